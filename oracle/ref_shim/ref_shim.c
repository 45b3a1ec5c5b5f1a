/* Project-written stand-ins for the libraries the reference links but this
 * repository cannot vendor: dedisp (always reports an error), a file-backed
 * psrdada reader, and getVDIFDMJD restated from the VDIF specification
 * (epoch = 6-month periods since 2000-01-01; seconds from the epoch start).
 * Built with REF_SHIM_DADA_ONLY, only the psrdada reader stand-in (the tests
 * of the tools' psrdada input build it that way). */
#include <stdio.h>
#include <string.h>

#include "ipcio.h"
#ifndef REF_SHIM_DADA_ONLY
#include "dedisp.h"
#include "vdifio.h"

dedisp_error dedisp_set_device(int device) { (void)device; return DEDISP_NO_ERROR; }
const char* dedisp_get_error_string(dedisp_error e) { (void)e; return "dedisp library unavailable"; }
dedisp_error dedisp_create_plan(dedisp_plan* p, dedisp_size n, dedisp_float dt, dedisp_float f0, dedisp_float df) {
  (void)p; (void)n; (void)dt; (void)f0; (void)df; return 1;
}
dedisp_error dedisp_set_dm_list(dedisp_plan p, const dedisp_float* d, dedisp_size c) { (void)p; (void)d; (void)c; return 1; }
dedisp_size dedisp_get_dm_count(const dedisp_plan p) { (void)p; return 0; }
dedisp_size dedisp_get_max_delay(const dedisp_plan p) { (void)p; return 0; }
dedisp_error dedisp_execute(const dedisp_plan p, dedisp_size n, const dedisp_byte* i, dedisp_size ib, dedisp_byte* o,
                            dedisp_size ob, unsigned f) {
  (void)p; (void)n; (void)i; (void)ib; (void)o; (void)ob; (void)f; return 1;
}
void dedisp_destroy_plan(dedisp_plan p) { (void)p; }
#endif /* REF_SHIM_DADA_ONLY */

static char g_dada_path[4096];
static int g_iread = -1;
void ref_shim_set_dada_file(const char* path) { strncpy(g_dada_path, path, sizeof(g_dada_path) - 1); }
/* the iread value a connect finds (a stale primary reader when != -1) */
void ref_shim_set_iread(int iread) { g_iread = iread; }
int ipcio_connect(ipcio_t* io, key_t key) { (void)key; memset(io, 0, sizeof(*io)); io->buf.iread = g_iread; return 0; }
int ipcio_open(ipcio_t* io, char rdwrt) {
  (void)rdwrt;
  io->buf.f = fopen(g_dada_path, "rb");
  return io->buf.f ? 0 : -1;
}
long ipcio_read(ipcio_t* io, char* buf, size_t n) {
  if (!io->buf.f) return -1;
  size_t r = fread(buf, 1, n, io->buf.f);
  io->buf.nread += r;
  if (r < n) io->buf.eod = 1;
  return (long)r;
}
int ipcio_close(ipcio_t* io) { if (io->buf.f) fclose(io->buf.f); io->buf.f = NULL; return 0; }
int ipcio_disconnect(ipcio_t* io) { (void)io; return 0; }
uint64_t ipcio_tell(ipcio_t* io) { return io->buf.nread; }
uint64_t ipcio_space_left(ipcio_t* io) { (void)io; return 0; }
float ipcio_percent_full(ipcio_t* io) { (void)io; return 0.f; }
int ipcbuf_eod(ipcbuf_t* b) { return b->eod; }
uint64_t ipcbuf_get_nbufs(ipcbuf_t* b) { (void)b; return 1; }
uint64_t ipcbuf_get_bufsz(ipcbuf_t* b) { (void)b; return 0; }
uint64_t ipcbuf_get_nfull(ipcbuf_t* b) { (void)b; return 0; }
uint64_t ipcbuf_get_nclear(ipcbuf_t* b) { (void)b; return 0; }
uint64_t ipcbuf_get_write_count(ipcbuf_t* b) { (void)b; return 0; }
uint64_t ipcbuf_get_read_count(ipcbuf_t* b) { return b->nread; }
int ipcbuf_get_nreaders(ipcbuf_t* b) { (void)b; return 1; }

#ifndef REF_SHIM_DADA_ONLY
/* days from 1970-01-01 of a Gregorian date */
static long days_from_civil(long y, unsigned m, unsigned d) {
  y -= m <= 2;
  const long era = (y >= 0 ? y : y - 399) / 400;
  const unsigned yoe = (unsigned)(y - era * 400);
  const unsigned doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
  const unsigned doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + (long)doe - 719468;
}
int getVDIFFrameMJD(const vdif_header* h) {
  const long mjd_epoch = days_from_civil(2000 + h->epoch / 2, 1 + 6 * (h->epoch % 2), 1) + 40587;
  return (int)(mjd_epoch + h->seconds / 86400);
}
double getVDIFDMJD(const vdif_header* h, int fps) {
  return getVDIFFrameMJD(h) + (double)getVDIFFrameSecond(h) / 86400.0 + (double)getVDIFFrameNumber(h) / (fps * 86400.0);
}
#endif /* REF_SHIM_DADA_ONLY */
