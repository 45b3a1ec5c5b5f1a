/* Minimal file-backed stand-in for psrdada's ipcio reader API as called by
 * the reference (STATS:284-304, 458-515; TS:355-389, 767-890).  The first
 * member is the ipcbuf_t, because the reference casts &ipcio_t to
 * ipcbuf_t*.  Project-written. */
#ifndef REF_SHIM_IPCIO_H
#define REF_SHIM_IPCIO_H
#include "ipcbuf.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct ipcio_t {
  ipcbuf_t buf;
} ipcio_t;
/* the harness names the file that stands in for the shared-memory ring */
void ref_shim_set_dada_file(const char* path);
/* the iread value the next ipcio_connect finds (-1 unless set) */
void ref_shim_set_iread(int iread);
int ipcio_connect(ipcio_t* io, key_t key);
int ipcio_open(ipcio_t* io, char rdwrt);
long ipcio_read(ipcio_t* io, char* buf, size_t n);
int ipcio_close(ipcio_t* io);
int ipcio_disconnect(ipcio_t* io);
uint64_t ipcio_tell(ipcio_t* io);
uint64_t ipcio_space_left(ipcio_t* io);
float ipcio_percent_full(ipcio_t* io);
#ifdef __cplusplus
}
#endif
#endif
