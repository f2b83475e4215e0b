/*
 * nf_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of the abacus near-field direct-force path, used only by
 * tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the
 * checker.  Nothing in the product library links or calls this file.
 *
 * Three computations live here:
 *
 *  1. nfo_ref32_slab(): the reference CPU direct, restated in plain C.
 *     It follows singlestep/Timestep/extras_directdriver.cpp:59-122
 *     (NearFieldDriver::ExecuteSlabCPU: 125 source cells per sink cell, the
 *     sink shifted by delta = CellCenter(sink) - CellCenter(source) computed
 *     in double and cast to float), singlestep/Direct/direct.cpp:49-59
 *     (Direct::Execute: per-source-cell FP32 partial, then SA[q] += acc) and
 *     singlestep/Direct/DirectCPUKernels.cc:12-129 (directkernel<0> for the
 *     four softenings, exact 1.0f/sqrtf).  Evaluation order follows the
 *     reference expression trees so that, built with -ffp-contract=off, it
 *     reproduces the reference compiled the same way bit for bit.
 *
 *  2. nfo_fp64_sinks(): an FP64 direct sum over the identical 5x5x5 cell
 *     neighbourhoods (the precision yardstick).  Global positions are
 *     (double)float32 local position + (double) cell offset; the softening
 *     formulas are the reference's, evaluated in double.
 *
 *  3. nfo_frame32_sinks(): a CPU model of the B200 kernel's arithmetic
 *     (cell-pair frames centred between the two cells, rsqrt + one Newton
 *     step, per-column FP32 partials folded into a compensated (hi, lo) sum).
 *     It lets the error budget of that arithmetic be studied on the CPU.
 *
 *  4. nfo_cpu_execute(): SetInteractionCollection::CPUExecute
 *     (singlestep/Direct/extras_PencilOnPencil.cc:7-152), the reference's CPU
 *     twin of the GPU pencil kernel (Plummer only, as there): every padded
 *     sink slot of every 64-sink block against the 2R+1 source pencils of its
 *     interaction list, y offset added per interaction, FP32 throughout.  It
 *     runs on the SIC arrays oracle.py builds in the reference's layout, so it
 *     pins the pencil decomposition itself against the cell-loop direct.
 *
 * Data layout (shared with the product library): a periodic unit box of
 * cpd^3 cells (cpd odd), particles sorted by cell id ((cx*cpd)+cy)*cpd+cz,
 * positions as three float32 arrays relative to the cell centre,
 * cell_start[cpd^3+1] prefix offsets.  Accelerations are written as three
 * floats per particle (x,y,z), at the particle's index.
 *
 * Softening ids: 0 Plummer, 1 single spline, 2 cubic spline, 3 cubic Plummer.
 * "eps" is the reference's kernel parameter (directdriver.cpp:109-117):
 * eps^2, 1/eps^2, 1/eps, eps^3 respectively.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NFO_PLUMMER 0
#define NFO_SINGLE_SPLINE 1
#define NFO_CUBIC_SPLINE 2
#define NFO_CUBIC_PLUMMER 3

/* The reference writes RSQRT as `1.0f/sqrt` (DirectCPUKernels.cc:8) with only
 * <cmath> in scope, where the unqualified call resolves to the C library's
 * double sqrt: the reciprocal square root is formed in double and rounded to
 * float once, on assignment. */
static inline float rsqrt_ref(float v) { return (float)(1.0f / sqrt((double)v)); }

static inline int wrapi(int i, int cpd) {
    while (i >= cpd) i -= cpd;
    while (i < 0) i += cpd;
    return i;
}

/* ---------------------------------------------------------------------- */
/* 1. reference FP32 CPU direct                                            */
/* ---------------------------------------------------------------------- */

/* directkernel<0>, DirectCPUKernels.cc:109-128 (default Plummer). */
static inline void k32_plummer(const float s[3], float tx, float ty, float tz,
                               float a[3], float eps2) {
    float drx = tx - s[0], dry = ty - s[1], drz = tz - s[2];
    float r = rsqrt_ref(drx * drx + dry * dry + drz * drz + eps2);
    r *= r * r;
    a[0] -= r * drx;
    a[1] -= r * dry;
    a[2] -= r * drz;
}

/* directkernel<0>, DirectCPUKernels.cc:53-80 (single spline, R<=1 branch). */
static inline void k32_single_spline(const float s[3], float tx, float ty, float tz,
                                     float a[3], float inv_eps2) {
    float dx = tx - s[0], dy = ty - s[1], dz = tz - s[2];
    float dr2 = (dx * dx + dy * dy + dz * dz) * inv_eps2 + (float)1e-32;
    float f = rsqrt_ref(dr2);
    f = fminf(f * f * f, (-15 * f + 6) * dr2 + 10);
    a[0] -= f * dx;
    a[1] -= f * dy;
    a[2] -= f * dz;
}

/* directkernel<0>, DirectCPUKernels.cc:12-51 (Hernquist & Katz cubic spline). */
static inline void k32_cubic_spline(const float s[3], float tx, float ty, float tz,
                                    float a[3], float eps_inv) {
    float drx = tx - s[0], dry = ty - s[1], drz = tz - s[2];
    float rinv = rsqrt_ref(drx * drx + dry * dry + drz * drz);
    float u = eps_inv / rinv, spf;
    if (u >= (float)(2.0))
        spf = rinv * rinv * rinv;
    else if (u >= (float)(1.0))
        spf = rinv * rinv * rinv *
              ((float)(-1.0 / 15.0) + (float)(8.0 / 3.0) * u * u * u -
               (float)(3.0) * u * u * u * u + (float)(6.0 / 5.0) * u * u * u * u * u -
               (float)(1.0 / 6.0) * u * u * u * u * u * u);
    else
        spf = eps_inv * eps_inv * eps_inv *
              ((float)(4.0 / 3.0) - (float)(6.0 / 5.0) * u * u + (float)(1.0 / 2.0) * u * u * u);
    a[0] -= spf * drx;
    a[1] -= spf * dry;
    a[2] -= spf * drz;
}

/* directkernel<0>, DirectCPUKernels.cc:82-106 (cubic Plummer, TAU2 = 1e-16). */
static inline void k32_cubic_plummer(const float s[3], float tx, float ty, float tz,
                                     float a[3], float eps3) {
    float drx = tx - s[0], dry = ty - s[1], drz = tz - s[2];
    float r = drx * drx + dry * dry + drz * drz + (float)(1e-16);
    /* `r *= r*RSQRT(r)` expands to r *= r*1.0f/sqrt(r): a double quotient
     * r/sqrt(r), a double product, one rounding to float on assignment. */
    r = (float)((double)r * ((double)r / sqrt((double)r)));
    r += eps3;
    r = (float)(1.0) / r;
    a[0] -= r * drx;
    a[1] -= r * dry;
    a[2] -= r * drz;
}

/* Direct::Execute (direct.cpp:49-59) for one (sink cell, source cell) pair:
 * acc = 0; sink = delta + sinks[q]; for p: kernel; SA[q] += acc. */
static void ref32_execute(int soft, const float *sx, const float *sy, const float *sz, int64_t ns,
                          const float *tx, const float *ty, const float *tz, int64_t nt,
                          const float delta[3], float eps, float *SA) {
    for (int64_t q = 0; q < ns; q++) {
        float acc[3] = {0.f, 0.f, 0.f};
        float sink[3] = {delta[0] + sx[q], delta[1] + sy[q], delta[2] + sz[q]};
        switch (soft) {
        case NFO_PLUMMER:
            for (int64_t p = 0; p < nt; p++) k32_plummer(sink, tx[p], ty[p], tz[p], acc, eps);
            break;
        case NFO_SINGLE_SPLINE:
            for (int64_t p = 0; p < nt; p++) k32_single_spline(sink, tx[p], ty[p], tz[p], acc, eps);
            break;
        case NFO_CUBIC_SPLINE:
            for (int64_t p = 0; p < nt; p++) k32_cubic_spline(sink, tx[p], ty[p], tz[p], acc, eps);
            break;
        default:
            for (int64_t p = 0; p < nt; p++) k32_cubic_plummer(sink, tx[p], ty[p], tz[p], acc, eps);
            break;
        }
        SA[3 * q + 0] += acc[0];
        SA[3 * q + 1] += acc[1];
        SA[3 * q + 2] += acc[2];
    }
}

/* NearFieldDriver::ExecuteSlabCPU (extras_directdriver.cpp:59-122) for one
 * sink cell (x,y,z): zero its accelerations, then loop i (x), j (y), k (z)
 * over the 5x5x5 neighbourhood in that order.  acc is indexed by particle. */
static void ref32_cell(int cpd, int R, const int64_t *cs, const float *x, const float *y,
                       const float *z, int soft, float eps, int cx, int cy, int cz, float *acc) {
    int64_t c = ((int64_t)cx * cpd + cy) * cpd + cz;
    int64_t s0 = cs[c], ns = cs[c + 1] - cs[c];
    float *SA = acc + 3 * s0;
    memset(SA, 0, sizeof(float) * 3 * (size_t)ns);
    if (ns == 0) return;
    double invcpd = 1.0 / (double)cpd;
    int cpdhalf = (cpd - 1) / 2;
    for (int i = cx - R; i <= cx + R; i++)
        for (int j = cy - R; j <= cy + R; j++)
            for (int k = cz - R; k <= cz + R; k++) {
                int64_t t = ((int64_t)wrapi(i, cpd) * cpd + wrapi(j, cpd)) * cpd + wrapi(k, cpd);
                int64_t t0 = cs[t], nt = cs[t + 1] - cs[t];
                if (nt <= 0) continue;
                /* CellCenter is not wrapped (grid.cpp:92-96); the difference
                 * is taken in double and cast to FLOAT3. */
                float delta[3] = {
                    (float)((cx - cpdhalf) * invcpd - (i - cpdhalf) * invcpd),
                    (float)((cy - cpdhalf) * invcpd - (j - cpdhalf) * invcpd),
                    (float)((cz - cpdhalf) * invcpd - (k - cpdhalf) * invcpd)};
                ref32_execute(soft, x + s0, y + s0, z + s0, ns, x + t0, y + t0, z + t0, nt, delta,
                              eps, SA);
            }
}

/* One x-slab, all sink cells, OpenMP over y as in the reference. */
int nfo_ref32_slab(int cpd, int R, const int64_t *cell_start, const float *x, const float *y,
                   const float *z, int soft, float eps, int slab, float *acc) {
    if (cpd <= 0 || (cpd & 1) == 0 || R < 0 || 2 * R + 1 > cpd || slab < 0 || slab >= cpd)
        return -1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int yy = 0; yy < cpd; yy++)
        for (int zz = 0; zz < cpd; zz++)
            ref32_cell(cpd, R, cell_start, x, y, z, soft, eps, slab, yy, zz, acc);
    return 0;
}

/* Same, for an explicit list of sink cells (linear ids). */
int nfo_ref32_cells(int cpd, int R, const int64_t *cell_start, const float *x, const float *y,
                    const float *z, int soft, float eps, const int64_t *cells, int64_t ncells,
                    float *acc) {
    if (cpd <= 0 || (cpd & 1) == 0 || R < 0 || 2 * R + 1 > cpd) return -1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t n = 0; n < ncells; n++) {
        int64_t c = cells[n];
        int cz = (int)(c % cpd), cy = (int)((c / cpd) % cpd), cx = (int)(c / ((int64_t)cpd * cpd));
        ref32_cell(cpd, R, cell_start, x, y, z, soft, eps, cx, cy, cz, acc);
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* 2. FP64 oracle                                                          */
/* ---------------------------------------------------------------------- */

static int64_t cell_of(const int64_t *cs, int64_t ncell, int64_t p) {
    /* largest c with cs[c] <= p and cs[c+1] > p */
    int64_t lo = 0, hi = ncell; /* cs[lo] <= p < cs[hi] */
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) / 2;
        if (cs[mid] <= p) lo = mid; else hi = mid;
    }
    return lo;
}

/* g(r^2) such that a = -sum g * d, in the reference's raw output units. */
static inline double k64(int soft, double r2, double eps) {
    switch (soft) {
    case NFO_PLUMMER: {
        double r = 1.0 / sqrt(r2 + eps);
        return r * r * r;
    }
    case NFO_SINGLE_SPLINE: {
        double dr2 = r2 * eps + 1e-32;
        double f = 1.0 / sqrt(dr2);
        double far = f * f * f, near = (-15.0 * f + 6.0) * dr2 + 10.0;
        return far < near ? far : near;
    }
    case NFO_CUBIC_SPLINE: {
        if (r2 == 0.0) return 0.0;
        double rinv = 1.0 / sqrt(r2);
        double u = eps / rinv;
        if (u >= 2.0) return rinv * rinv * rinv;
        if (u >= 1.0)
            return rinv * rinv * rinv *
                   (-1.0 / 15.0 + 8.0 / 3.0 * u * u * u - 3.0 * u * u * u * u +
                    6.0 / 5.0 * u * u * u * u * u - 1.0 / 6.0 * u * u * u * u * u * u);
        return eps * eps * eps * (4.0 / 3.0 - 6.0 / 5.0 * u * u + 0.5 * u * u * u);
    }
    default: {
        double r = r2 + 1e-16;
        r = r * sqrt(r) + eps;
        return 1.0 / r;
    }
    }
}

/* FP64 acceleration of the listed sink particles (global indices), summed
 * over the 5x5x5 cells around each sink's cell.  eps as for the FP32 path
 * (pass (double) of the float value to measure exactly that function). */
int nfo_fp64_sinks(int cpd, int R, const int64_t *cell_start, const float *x, const float *y,
                   const float *z, int soft, double eps, const int64_t *sinks, int64_t nsinks,
                   double *acc) {
    if (cpd <= 0 || (cpd & 1) == 0 || R < 0 || 2 * R + 1 > cpd) return -1;
    int64_t ncell = (int64_t)cpd * cpd * cpd;
    double h = 1.0 / (double)cpd;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t n = 0; n < nsinks; n++) {
        int64_t p = sinks[n];
        int64_t c = cell_of(cell_start, ncell, p);
        int cz = (int)(c % cpd), cy = (int)((c / cpd) % cpd), cx = (int)(c / ((int64_t)cpd * cpd));
        double sx = x[p], sy = y[p], sz = z[p];
        double ax = 0, ay = 0, az = 0;
        for (int dx = -R; dx <= R; dx++)
            for (int dy = -R; dy <= R; dy++)
                for (int dz = -R; dz <= R; dz++) {
                    int64_t t = ((int64_t)wrapi(cx + dx, cpd) * cpd + wrapi(cy + dy, cpd)) * cpd +
                                wrapi(cz + dz, cpd);
                    double ox = dx * h, oy = dy * h, oz = dz * h;
                    for (int64_t q = cell_start[t]; q < cell_start[t + 1]; q++) {
                        double ddx = ((double)x[q] - sx) + ox;
                        double ddy = ((double)y[q] - sy) + oy;
                        double ddz = ((double)z[q] - sz) + oz;
                        double g = k64(soft, ddx * ddx + ddy * ddy + ddz * ddz, eps);
                        ax -= g * ddx;
                        ay -= g * ddy;
                        az -= g * ddz;
                    }
                }
        acc[3 * n + 0] = ax;
        acc[3 * n + 1] = ay;
        acc[3 * n + 2] = az;
    }
    return 0;
}

/* Exact pair count (DirectTotal): sum over sink cells of n_sink * sum of the
 * 125 neighbour counts (PencilOnPencil.cc:412, DirectBench.cpp:111-125). */
uint64_t nfo_pair_count(int cpd, int R, const int64_t *cell_start) {
    uint64_t total = 0;
#pragma omp parallel for reduction(+ : total) schedule(static)
    for (int cx = 0; cx < cpd; cx++)
        for (int cy = 0; cy < cpd; cy++)
            for (int cz = 0; cz < cpd; cz++) {
                int64_t c = ((int64_t)cx * cpd + cy) * cpd + cz;
                uint64_t ns = (uint64_t)(cell_start[c + 1] - cell_start[c]);
                if (!ns) continue;
                uint64_t nsrc = 0;
                for (int dx = -R; dx <= R; dx++)
                    for (int dy = -R; dy <= R; dy++)
                        for (int dz = -R; dz <= R; dz++) {
                            int64_t t = ((int64_t)wrapi(cx + dx, cpd) * cpd + wrapi(cy + dy, cpd)) *
                                            cpd + wrapi(cz + dz, cpd);
                            nsrc += (uint64_t)(cell_start[t + 1] - cell_start[t]);
                        }
                total += ns * nsrc;
            }
    return total;
}

/* ---------------------------------------------------------------------- */
/* 3. CPU model of the B200 kernel arithmetic                              */
/* ---------------------------------------------------------------------- */

/* rsqrt plus one Newton-Raphson step, applied to the cube:
 *   y = rsqrt(r2); e = r2*y^2 - 1; f = y^3 * (1 - 1.5 e)
 * (first-order Newton correction of y, cubed).  Here y comes from the
 * correctly rounded 1/sqrtf, which only models the hardware estimate. */
static inline float newton_cube(float r2) {
    float y = 1.0f / sqrtf(r2);
    float y2 = y * y;
    float y3 = y2 * y;
    float e = fmaf(r2, y2, -1.0f);
    float g = y3 * e;
    return fmaf(g, -1.5f, y3);
}

static inline void two_sum(float a, float b, float *s, float *err) {
    float ss = a + b;
    float bb = ss - a;
    *err = (a - (ss - bb)) + (b - bb);
    *s = ss;
}

/* Cell-pair frames: for a source cell offset n (per component), both sides
 * are moved to an origin half-way between the two cell centres:
 *   t_f = t + n*H ,  s_f = (s - n*H) - n*L ,  H = fl(h/2), L = fl(h - 2H)
 * so that t_f - s_f = t - s + n*h to within the rounding of t_f and s_f,
 * whose magnitudes are the distances to that origin.  Each 5-cell column's
 * FP32 partial is folded into a (hi, lo) TwoSum pair when compensated.
 * The spline result is accumulated as sum g*d with g = r^-3 (far) or
 * f_spline * eps^-3 (near, exact reference formula) and scaled by eps^3
 * once at the end.
 *
 * flags (for error-budget studies):
 *   1  compensated column partials (else plain FP32 running sum)
 *   2  reference frame instead: sink + fl(CellCenter(s) - CellCenter(t))
 *   4  reference pair value: r = fl(1/sqrt(r2)), g = r*r*r
 *   8  partials per source cell instead of per 5-cell column
 *  16  a -= g*d as multiply then subtract (else one fused multiply-add)
 *  32  g evaluated in double from the float32 differences
 *  64  accumulate in double (isolates the pair-evaluation error)
 *  bits 8..23: if nonzero, also fold the partial every that many sources
 */
int nfo_frame32_sinks(int cpd, int R, const int64_t *cell_start, const float *x, const float *y,
                      const float *z, int soft, float eps, int flags, const int64_t *sinks,
                      int64_t nsinks, float *acc) {
    if (cpd <= 0 || (cpd & 1) == 0 || R < 0 || 2 * R + 1 > cpd) return -1;
    if (soft != NFO_PLUMMER && soft != NFO_SINGLE_SPLINE) return -2;
    int64_t ncell = (int64_t)cpd * cpd * cpd;
    double h = 1.0 / (double)cpd;
    float H = (float)(0.5 * h);
    float L = (float)(h - 2.0 * (double)H);
    /* single spline: eps = 1/eps_int^2 */
    double e_int = soft == NFO_SINGLE_SPLINE ? 1.0 / sqrt((double)eps) : 0.0;
    float eps2_unscaled = (float)(e_int * e_int);
    float near_thr = eps2_unscaled * 1.0001f;
    float eps3 = (float)(e_int * e_int * e_int);
    float inv_eps3 = (float)(1.0 / (e_int * e_int * e_int));
    int cpdhalf = (cpd - 1) / 2;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t n = 0; n < nsinks; n++) {
        int64_t p = sinks[n];
        int64_t c = cell_of(cell_start, ncell, p);
        int cz = (int)(c % cpd), cy = (int)((c / cpd) % cpd), cx = (int)(c / ((int64_t)cpd * cpd));
        float hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0};
        float part[3] = {0, 0, 0};
        double dacc[3] = {0, 0, 0};
        int chunk = (flags >> 8) & 0xffff, inchunk = 0;
        for (int dx = -R; dx <= R; dx++)
            for (int dy = -R; dy <= R; dy++) {
                for (int dz = -R; dz <= R; dz++) {
                    int off[3] = {dx, dy, dz};
                    float sf[3], sh[3];
                    float s[3] = {x[p], y[p], z[p]};
                    for (int k = 0; k < 3; k++) {
                        sh[k] = (float)off[k] * H;  /* exact: |off| <= 2 */
                        if (flags & 2) {
                            int ci = k == 0 ? cx : k == 1 ? cy : cz;
                            float delta = (float)((ci - cpdhalf) * h - (ci + off[k] - cpdhalf) * h);
                            sf[k] = delta + s[k];
                        } else {
                            sf[k] = off[k] ? (s[k] - sh[k]) - (float)off[k] * L : s[k];
                        }
                    }
                    int64_t t = ((int64_t)wrapi(cx + dx, cpd) * cpd + wrapi(cy + dy, cpd)) * cpd +
                                wrapi(cz + dz, cpd);
                    for (int64_t q = cell_start[t]; q < cell_start[t + 1]; q++) {
                        float tf0 = x[q], tf1 = y[q], tf2 = z[q];
                        if (!(flags & 2)) {
                            if (off[0]) tf0 += sh[0];
                            if (off[1]) tf1 += sh[1];
                            if (off[2]) tf2 += sh[2];
                        }
                        float d0 = tf0 - sf[0], d1 = tf1 - sf[1], d2 = tf2 - sf[2];
                        float g;
                        if (soft == NFO_PLUMMER) {
                            float r2 = fmaf(d2, d2, fmaf(d1, d1, fmaf(d0, d0, eps)));
                            if (flags & 32) {
                                double rr = (double)d0 * d0 + (double)d1 * d1 + (double)d2 * d2 + (double)eps;
                                g = (float)(1.0 / (rr * sqrt(rr)));
                            } else if (flags & 4) {
                                float r = rsqrt_ref(r2);
                                g = r * r * r;
                            } else {
                                g = newton_cube(r2);
                            }
                        } else {
                            float r2 = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
                            if (r2 < near_thr) {
                                float dr2 = fmaf(r2, eps, 1e-32f);
                                float f = 1.0f / sqrtf(dr2);
                                float f3 = f * f * f;
                                float pn = fmaf(fmaf(-15.0f, f, 6.0f), dr2, 10.0f);
                                g = (f3 < pn ? f3 : pn) * inv_eps3;
                            } else if (flags & 32) {
                                double rr = (double)d0 * d0 + (double)d1 * d1 + (double)d2 * d2;
                                g = (float)(1.0 / (rr * sqrt(rr)));
                            } else if (flags & 4) {
                                float r = rsqrt_ref(r2);
                                g = r * r * r;
                            } else {
                                g = newton_cube(r2);
                            }
                        }
                        if (flags & 64) {
                            dacc[0] -= (double)g * d0;
                            dacc[1] -= (double)g * d1;
                            dacc[2] -= (double)g * d2;
                        } else if (flags & 16) {
                            part[0] -= g * d0;
                            part[1] -= g * d1;
                            part[2] -= g * d2;
                        } else {
                            part[0] = fmaf(-g, d0, part[0]);
                            part[1] = fmaf(-g, d1, part[1]);
                            part[2] = fmaf(-g, d2, part[2]);
                        }
                        if (chunk && ++inchunk == chunk) {
                            inchunk = 0;
                            for (int k = 0; k < 3; k++) {
                                if (flags & 1) {
                                    float e;
                                    two_sum(hi[k], part[k], &hi[k], &e);
                                    lo[k] += e;
                                } else {
                                    hi[k] += part[k];
                                }
                                part[k] = 0.f;
                            }
                        }
                    }
                    int flush = (flags & 8) || dz == R;
                    if (flush) {
                        for (int k = 0; k < 3; k++) {
                            if (flags & 1) {
                                float e;
                                two_sum(hi[k], part[k], &hi[k], &e);
                                lo[k] += e;
                            } else {
                                hi[k] += part[k];
                            }
                            part[k] = 0.f;
                        }
                    }
                }
            }
        for (int k = 0; k < 3; k++) {
            float v = (flags & 64) ? (float)dacc[k] : hi[k] + lo[k];
            acc[3 * n + k] = soft == NFO_SINGLE_SPLINE ? v * eps3 : v;
        }
    }
    return 0;
}

/* FP64 FOF density channel of the listed sinks: w = sum over the 5x5x5
 * neighbourhood of (b2 - r^2) for r^2 < b2, r unsoftened
 * (singlestep/Direct/DirectGPUKernels.cuh:37-39, 85-88, 130-132, 162-164). */
int nfo_fp64_density(int cpd, int R, const int64_t *cell_start, const float *x, const float *y,
                     const float *z, double b2, const int64_t *sinks, int64_t nsinks, double *w) {
    if (cpd <= 0 || (cpd & 1) == 0 || R < 0 || 2 * R + 1 > cpd) return -1;
    int64_t ncell = (int64_t)cpd * cpd * cpd;
    double h = 1.0 / (double)cpd;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t n = 0; n < nsinks; n++) {
        int64_t p = sinks[n];
        int64_t c = cell_of(cell_start, ncell, p);
        int cz = (int)(c % cpd), cy = (int)((c / cpd) % cpd), cx = (int)(c / ((int64_t)cpd * cpd));
        double acc = 0;
        for (int dx = -R; dx <= R; dx++)
            for (int dy = -R; dy <= R; dy++)
                for (int dz = -R; dz <= R; dz++) {
                    int64_t t = ((int64_t)wrapi(cx + dx, cpd) * cpd + wrapi(cy + dy, cpd)) * cpd +
                                wrapi(cz + dz, cpd);
                    for (int64_t q = cell_start[t]; q < cell_start[t + 1]; q++) {
                        double ddx = ((double)x[q] - x[p]) + dx * h;
                        double ddy = ((double)y[q] - y[p]) + dy * h;
                        double ddz = ((double)z[q] - z[p]) + dz * h;
                        double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        if (r2 < b2) acc += b2 - r2;
                    }
                }
        w[n] = acc;
    }
    return 0;
}

/* SetInteractionCollection::CPUExecute (extras_PencilOnPencil.cc:7-152).
 * sink_xyz: X | Y | Z of nslots padded sink slots (z already shifted by
 * (c-R) h per sink cell, PencilPlan.cc:22-90); src_xyz: X | Y | Z of nsrc
 * sources (x shifted by (c-R) h per source cell, PencilPlan.cc:214-255);
 * id_max[p]: one past the last live slot of sink pencil p; parent[b]: the
 * pencil of block b; ilist / yoff: W source pencils and y offsets per sink
 * pencil; eps2 = eps_int^2 (cpu_eps).  acc: 3 floats per slot, written for
 * live slots only (extras_PencilOnPencil.cc:123-133). */
int nfo_cpu_execute(int nblocks, int nslots, const float *sink_xyz, const uint32_t *id_max,
                    const int32_t *parent, int nsrc, const float *src_xyz,
                    const int32_t *src_start, const int32_t *src_count, const int32_t *ilist,
                    const float *yoff, int W, float eps2, float *acc) {
    if (nblocks < 0 || nslots < 64 * nblocks || W < 1) return -1;
    const float *SX = sink_xyz, *SY = sink_xyz + nslots, *SZ = sink_xyz + 2 * (size_t)nslots;
    const float *TX = src_xyz, *TY = src_xyz + nsrc, *TZ = src_xyz + 2 * (size_t)nsrc;
    for (int b = 0; b < nblocks; b++) {
        const int p = parent[b];
        for (int t = 0; t < 64; t++) {
            const int64_t id = 64 * (int64_t)b + t;
            if (id >= (int64_t)id_max[p]) continue; /* padded slot: nothing stored */
            const float sinkX = SX[id], sinkY = SY[id], sinkZ = SZ[id];
            float ax = 0.f, ay = 0.f, az = 0.f;
            for (int c = p * W; c < p * W + W; c++) {
                const int s = ilist[c];
                const int st = src_start[s], n = src_count[s];
                const float yoffset = yoff[c];
                if (st < 0 || n < 0 || (int64_t)st + n > nsrc) return -2;
                for (int i = 0; i < n; i++) {
                    float drx = TX[st + i] - sinkX;
                    float dry = TY[st + i] - sinkY + yoffset;
                    float drz = TZ[st + i] - sinkZ;
                    /* (FLOAT)1./std::sqrt(float): the float overload */
                    float r = 1.0f / sqrtf(drx * drx + dry * dry + drz * drz + eps2);
                    r *= r * r;
                    ax -= r * drx;
                    ay -= r * dry;
                    az -= r * drz;
                }
            }
            acc[3 * id] = ax;
            acc[3 * id + 1] = ay;
            acc[3 * id + 2] = az;
        }
    }
    return 0;
}
