/* Minimal file-backed stand-in for the psrdada ring-buffer types the
 * reference touches (STATS:123-134, 292-304; TS:136-147, 366-382).
 * Only `iread` is read by the reference itself.  Project-written. */
#ifndef REF_SHIM_IPCBUF_H
#define REF_SHIM_IPCBUF_H
#include <stdint.h>
#include <stdio.h>
#include <sys/types.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct ipcbuf_t {
  int iread;
  FILE* f;
  int eod;
  uint64_t nread;
} ipcbuf_t;
int ipcbuf_eod(ipcbuf_t* b);
uint64_t ipcbuf_get_nbufs(ipcbuf_t* b);
uint64_t ipcbuf_get_bufsz(ipcbuf_t* b);
uint64_t ipcbuf_get_nfull(ipcbuf_t* b);
uint64_t ipcbuf_get_nclear(ipcbuf_t* b);
uint64_t ipcbuf_get_write_count(ipcbuf_t* b);
uint64_t ipcbuf_get_read_count(ipcbuf_t* b);
int ipcbuf_get_nreaders(ipcbuf_t* b);
#ifdef __cplusplus
}
#endif
#endif
