/* Stand-in declarations for the dedisp library API the reference calls
 * (PIPE:28, 202-218, 416-444, 671, 790).  The library itself is not
 * available here; the stand-in functions (ref_shim.c) report an error, and
 * the harness never calls the reference's main().  Project-written. */
#ifndef REF_SHIM_DEDISP_H
#define REF_SHIM_DEDISP_H
#ifdef __cplusplus
extern "C" {
#endif
typedef struct dedisp_plan_struct* dedisp_plan;
typedef unsigned long dedisp_size;
typedef float dedisp_float;
typedef unsigned char dedisp_byte;
typedef int dedisp_error;
#define DEDISP_NO_ERROR 0
#define DEDISP_DEVICE_POINTERS 1
dedisp_error dedisp_set_device(int device);
const char* dedisp_get_error_string(dedisp_error e);
dedisp_error dedisp_create_plan(dedisp_plan* plan, dedisp_size nchans, dedisp_float dt, dedisp_float f0,
                                dedisp_float df);
dedisp_error dedisp_set_dm_list(dedisp_plan plan, const dedisp_float* dms, dedisp_size count);
dedisp_size dedisp_get_dm_count(const dedisp_plan plan);
dedisp_size dedisp_get_max_delay(const dedisp_plan plan);
dedisp_error dedisp_execute(const dedisp_plan plan, dedisp_size nsamps, const dedisp_byte* in, dedisp_size in_nbits,
                            dedisp_byte* out, dedisp_size out_nbits, unsigned flags);
void dedisp_destroy_plan(dedisp_plan plan);
#ifdef __cplusplus
}
#endif
#endif
