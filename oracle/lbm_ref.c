/*
 * ORACLE — test infrastructure only. Never part of the product path.
 *
 * CPU restatement of tgautam03/xAdvCool's coupled D3Q19 fluid + thermal
 * lattice-Boltzmann path (src/fluid_engine3d.py, src/thermal_engine3d.py,
 * src/simulation.py and the test-only kernels of validate_analytical.py).
 * Built twice from lbm_ref_body.h: ref32_* (float, the parity oracle) and
 * ref64_* (double, the FP64 oracle for 16-bit storage error studies).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* src/fluid_engine3d.py:11-14 */
enum { BC_FLUID = 0, BC_SOLID = 1, BC_INLET = 2, BC_OUTLET = 3 };

/* src/fluid_engine3d.py:19-39: rest, 6 faces, 12 edges */
static const int E[19][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                             {1, 1, 0},  {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 0, 1},  {-1, 0, -1}, {1, 0, -1},
                             {-1, 0, 1}, {0, 1, 1},  {0, -1, -1}, {0, 1, -1}, {0, -1, 1}};
/* src/fluid_engine3d.py:51-53 */
static const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};

/* src/fluid_engine3d.py:42-47: weights are Python doubles rounded once to the storage type */
#define W_INIT(T)                                                                                              \
    {(T)(1.0 / 3.0),  (T)(1.0 / 18.0), (T)(1.0 / 18.0), (T)(1.0 / 18.0), (T)(1.0 / 18.0), (T)(1.0 / 18.0),   \
     (T)(1.0 / 18.0), (T)(1.0 / 36.0), (T)(1.0 / 36.0), (T)(1.0 / 36.0), (T)(1.0 / 36.0), (T)(1.0 / 36.0),   \
     (T)(1.0 / 36.0), (T)(1.0 / 36.0), (T)(1.0 / 36.0), (T)(1.0 / 36.0), (T)(1.0 / 36.0), (T)(1.0 / 36.0),   \
     (T)(1.0 / 36.0)}
static const float W32[19] = W_INIT(float);
static const double W64[19] = W_INIT(double);

#define REAL float
#define WR W32
#define PFX(name) ref32_##name
#include "lbm_ref_body.h"
#undef REAL
#undef WR
#undef PFX

#define REAL double
#define WR W64
#define PFX(name) ref64_##name
#include "lbm_ref_body.h"
#undef REAL
#undef WR
#undef PFX

int ref_num_threads(void)
{
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
