/* ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Drives the reference's own Direct::Execute (singlestep/Direct/direct.cpp,
 * compiled unmodified from its sources next to this file) with a re-hosting
 * of NearFieldDriver::ExecuteSlabCPU's cell loop
 * (singlestep/Timestep/extras_directdriver.cpp:59-122): OpenMP over y,
 * one Direct object per thread, for every sink cell zero its accelerations,
 * then for i, j, k over the 5x5x5 neighbourhood copy the source cell into
 * AoS, form delta = CellCenter(sink) - CellCenter(source) in double, cast it
 * to FLOAT3 and call Execute.  The abacus slab/arena globals (CP, SB, SS) are
 * replaced by the flat cell-sorted layout used everywhere in this repository
 * (float32 x[], y[], z[] cell-relative; cell_start[cpd^3+1]).
 */
#include <omp.h>
#include <vector>
#include "direct.h"

static inline int wrapi(int i, int cpd) {
    while (i >= cpd) i -= cpd;
    while (i < 0) i += cpd;
    return i;
}

static void cell_loop(int cpd, int R, const int64_t *cs, const float *x, const float *y,
                      const float *z, float eps, int cx, int cy, int cz, float *acc,
                      Direct &D, std::vector<float3> &sinkbuf, std::vector<float3> &srcbuf) {
    int64_t c = ((int64_t)cx * cpd + cy) * cpd + cz;
    int64_t s0 = cs[c], ns = cs[c + 1] - cs[c];
    float3 *SA = (float3 *)(acc + 3 * s0);
    for (int64_t q = 0; q < ns; q++) SA[q] = float3(0.f, 0.f, 0.f);
    if (ns == 0) return;
    sinkbuf.resize(ns);
    for (int64_t q = 0; q < ns; q++) sinkbuf[q] = float3(x[s0 + q], y[s0 + q], z[s0 + q]);
    double invcpd = 1.0 / (double)cpd;   /* grid.cpp:44 */
    int cpdhalf = (cpd - 1) / 2;
    for (int i = cx - R; i <= cx + R; i++)
        for (int j = cy - R; j <= cy + R; j++)
            for (int k = cz - R; k <= cz + R; k++) {
                int64_t t = ((int64_t)wrapi(i, cpd) * cpd + wrapi(j, cpd)) * cpd + wrapi(k, cpd);
                int64_t t0 = cs[t], nt = cs[t + 1] - cs[t];
                srcbuf.resize(nt > 0 ? nt : 1);
                for (int64_t q = 0; q < nt; q++)
                    srcbuf[q] = float3(x[t0 + q], y[t0 + q], z[t0 + q]);
                double3 cs_ = {(cx - cpdhalf) * invcpd, (cy - cpdhalf) * invcpd, (cz - cpdhalf) * invcpd};
                double3 ct_ = {(i - cpdhalf) * invcpd, (j - cpdhalf) * invcpd, (k - cpdhalf) * invcpd};
                FLOAT3 delta = cs_ - ct_;
                if (nt > 0)
                    D.AVXExecute(sinkbuf.data(), srcbuf.data(), (int)ns, (int)nt, delta, eps, SA);
            }
}

extern "C" int nfref_max_threads(void) { return omp_get_max_threads(); }

extern "C" int nfref_execute_slab(int cpd, int R, const int64_t *cs, const float *x,
                                  const float *y, const float *z, float eps, int slab,
                                  float *acc, int threads) {
    if (cpd <= 0 || (cpd & 1) == 0 || R < 0 || 2 * R + 1 > cpd || slab < 0 || slab >= cpd)
        return -1;
    int nt = threads > 0 ? threads : omp_get_max_threads();
    std::vector<Direct> DD(nt);
#pragma omp parallel num_threads(nt)
    {
        std::vector<float3> sinkbuf, srcbuf;
        int g = omp_get_thread_num();
#pragma omp for schedule(dynamic, 1)
        for (int yy = 0; yy < cpd; yy++)
            for (int zz = 0; zz < cpd; zz++)
                cell_loop(cpd, R, cs, x, y, z, eps, slab, yy, zz, acc, DD[g], sinkbuf, srcbuf);
    }
    return 0;
}

extern "C" int nfref_execute_cells(int cpd, int R, const int64_t *cs, const float *x,
                                   const float *y, const float *z, float eps,
                                   const int64_t *cells, int64_t ncells, float *acc,
                                   int threads) {
    if (cpd <= 0 || (cpd & 1) == 0 || R < 0 || 2 * R + 1 > cpd) return -1;
    int nt = threads > 0 ? threads : omp_get_max_threads();
    std::vector<Direct> DD(nt);
#pragma omp parallel num_threads(nt)
    {
        std::vector<float3> sinkbuf, srcbuf;
        int g = omp_get_thread_num();
#pragma omp for schedule(dynamic, 1)
        for (int64_t n = 0; n < ncells; n++) {
            int64_t c = cells[n];
            int cz = (int)(c % cpd), cy = (int)((c / cpd) % cpd);
            int cx = (int)(c / ((int64_t)cpd * cpd));
            cell_loop(cpd, R, cs, x, y, z, eps, cx, cy, cz, acc, DD[g], sinkbuf, srcbuf);
        }
    }
    return 0;
}
