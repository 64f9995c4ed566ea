/* keepsake-b200: C ABI of the B200-native small_pt path tracer.
 *
 * The entry points replace the parts of keepsake's CPU `small_pt` path that a C/C++ host calls
 * (reference interfaces cited per function).  Plain C types only; every call returns a
 * ks_status and never aborts; host pointers unless a name says `device`.
 *
 * Threading: a context owns one CUDA stream.  Calls on one context must not overlap; distinct
 * contexts may be used from distinct threads.
 */
#ifndef KS_B200_H
#define KS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ks_status {
    KS_OK = 0,
    KS_ERR_INVALID_ARGUMENT = 1,
    KS_ERR_OUT_OF_MEMORY = 2,
    KS_ERR_CUDA = 3,
    KS_ERR_QUEUE_OVERFLOW = 4,
    KS_ERR_WATCHDOG = 5,
    KS_ERR_NOT_BUILT = 6,
    KS_ERR_UNSUPPORTED = 7,
    KS_ERR_PARSE = 8,
    KS_ERR_IO = 9,
} ks_status;

typedef struct ks_context ks_context;

/* Context: one CUDA device + one stream.  (Replaces the reference's implicit global state:
 * EmbreeDevice in small_pt.cpp:182 and the TBB arena of parallel.h:93-113.) */
ks_status ks_context_create(int device, ks_context **out);
void ks_context_destroy(ks_context *ctx);
const char *ks_status_string(ks_status s);
/* Detail message of the last failing call on this context ("" if none). */
const char *ks_last_error(const ks_context *ctx);

/* Sobol parity hook.  For every pixel (x0..x0+nx-1, y0..y0+ny-1), sample index s0..s0+ns-1 and
 * dimension d in 0..nd-1 it starts a PTRenderSampler(full_res, pixel, spp, s, seed) at dimension d
 * (sobol.h:235-241 + start_pixel :140) and writes three floats:
 *   out[0] = sobol.next()   (sobol.h:148-156)
 *   out[1..2] = sobol.next2d() (sobol.h:158-167), each from a fresh sampler at dimension d.
 * Layout: out[(((py * nx + px) * ns + s) * nd + d) * 3 + c], host memory. */
ks_status ks_sobol_points(ks_context *ctx, uint32_t full_width, uint32_t full_height, uint32_t spp, uint32_t seed,
                          uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0, uint32_t ns, uint32_t nd,
                          float *out);

#ifdef __cplusplus
}
#endif

#endif /* KS_B200_H */
