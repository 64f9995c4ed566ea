// ORACLE (test infrastructure only).  C entry points of the CPU restatement, loaded by tests/
// and by bench.py's CPU-baseline leg through ctypes.  Nothing in the product links this library.
#include "o_sampler.h"

#include <cstdint>

extern "C" {

// Same contract and layout as ks_sobol_points() in include/ks_b200.h.
int oracle_sobol_points(uint32_t full_w, uint32_t full_h, uint32_t spp, uint32_t seed, uint32_t x0, uint32_t y0,
                        uint32_t nx, uint32_t ny, uint32_t s0, uint32_t ns, uint32_t nd, float *out)
{
    size_t i = 0;
    for (uint32_t py = 0; py < ny; ++py)
        for (uint32_t px = 0; px < nx; ++px)
            for (uint32_t s = 0; s < ns; ++s)
                for (uint32_t d = 0; d < nd; ++d, ++i) {
                    oracle::PTRenderSampler a(full_w, full_h, x0 + px, y0 + py, spp, s0 + s, seed);
                    a.sobol.dimension = (int)d;
                    oracle::PTRenderSampler b = a;
                    out[3 * i + 0] = a.sobol.next();
                    b.sobol.next2d(out[3 * i + 1], out[3 * i + 2]);
                }
    return 0;
}

// Columns of generator matrices 0 and 1 (2 x 52 uint32), for the golden-fixture check.
void oracle_sobol_matrices01(uint32_t *out)
{
    for (int i = 0; i < 2 * oracle::sobol_matrix_size; ++i)
        out[i] = oracle::sobol_matrices().m[i];
}

} // extern "C"
