/* ref_kick_shim.cpp -- TEST INFRASTRUCTURE ONLY (a checker, never the product).
 *
 * Compiles the reference's singlestep/Timestep/kick.cpp unmodified (it is
 * #included below) with the reference's own FLOAT3p1 (include/float3p1.cpp)
 * and ThreeVector (include/threevector.hh) types, so that
 * RescaleAndCoAddAcceleration (kick.cpp:72-107), KickSlab (kick.cpp:59-70)
 * and KickCell (kick.cpp:30-56) run exactly as the reference compiles them,
 * on caller-given arrays.  This file supplies only what the rest of
 * singlestep would around them: the slab buffer / slab size / cell lookups
 * (SB, SS, CP) over one slab of caller arrays, the parameters and state the
 * functions read (P, NFD, WriteState, the node's z range), the Cell and
 * cellinfo fields they touch, and NUMA_FOR as a plain loop (the non-NUMA
 * fallback of include/numa_for.h, without OpenMP: one thread, sequential
 * sums).  The softening (-DDIRECTSINGLESPLINE) and the density channel
 * (-DCOMPUTE_FOF_DENSITY) are chosen by the same macros as the reference
 * build.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "threevector.hh"

#define FLOAT float
#define FLOAT3 float3
typedef uint64_t uint64;

#include "float3p1.cpp"

using velstruct = FLOAT3;
using acc3struct = FLOAT3;
#ifdef COMPUTE_FOF_DENSITY
using accstruct = FLOAT3p1;
#else
using accstruct = FLOAT3;
#endif

#define NO_CLAUSE
#define FALLBACK_DYNAMIC dynamic
#define NUMA_FOR(I, START, END, CLAUSE, FALLBACK) for (int64_t I = START; I < END; I++)
#define NUMA_FOR_END

struct shim_cellinfo {
    float mean_square_velocity, max_component_velocity, max_component_acceleration;
};
struct shim_aux {
    float dens;
    void set_density(float d) { dens = d; }
};
struct Cell {
    velstruct *vel;
    accstruct *acc;
    shim_aux *aux;
    shim_cellinfo *ci;
    uint32_t n;
    uint32_t count() const { return n; }
};

enum { AccSlab = 0, FarAccSlab = 1 };

// One slab of caller arrays: cell c = y * cpd + z holds particles
// [cell_start[c], cell_start[c+1]).
static struct {
    int cpd;
    const int64_t *cell_start;
    velstruct *vel;
    accstruct *acc;
    acc3struct *far;
    shim_aux *aux;
    shim_cellinfo *ci;
    uint64 n;
} g;

struct ShimSlabBuffer {
    void *GetSlabPtr(int type, int) { return type == AccSlab ? (void *)g.acc : (void *)g.far; }
};
struct ShimSlabSize {
    uint64 size(int) { return g.n; }
};
struct ShimCellParticles {
    int cpd;
    Cell GetCell(int, int y, int z) {
        int64_t c = (int64_t)y * g.cpd + z, s = g.cell_start[c];
        Cell r;
        r.vel = g.vel + s;
        r.acc = g.acc + s;
        r.aux = g.aux ? g.aux + s : nullptr;
        r.ci = g.ci + c;
        r.n = (uint32_t)(g.cell_start[c + 1] - s);
        return r;
    }
};
static ShimSlabBuffer sb_;
static ShimSlabSize ss_;
static ShimCellParticles cp_;
static ShimSlabBuffer *SB = &sb_;
static ShimSlabSize *SS = &ss_;
static ShimCellParticles *CP = &cp_;
static struct {
    double Omega_M, Omega_Smooth;
    int64_t np;
    int MakeGlass;
} P;
static struct {
    double SofteningLengthInternal;
} nfd_;
static decltype(nfd_) *NFD = &nfd_;
static struct {
    float DensityKernelRad2;
} WriteState;
static int node_z_start = 0, node_z_size = 0;

#include "kick.cpp"

extern "C" int nfrefkick_acc_floats(void) { return (int)(sizeof(accstruct) / sizeof(float)); }

/* RescaleAndCoAddAcceleration on n particles: nacc (accstruct records,
 * updated in place) and facc (float3 records). */
extern "C" int nfrefkick_rescale(int64_t n, float *nacc, const float *facc, double omega_m,
                                 double omega_smooth, int64_t np, int make_glass,
                                 double softening_length_internal, float b2) {
    if (n < 0 || (n > 0 && (!nacc || !facc))) return -1;
    g.n = (uint64)n;
    g.acc = (accstruct *)nacc;
    g.far = (acc3struct *)facc;
    P.Omega_M = omega_m;
    P.Omega_Smooth = omega_smooth;
    P.np = np;
    P.MakeGlass = make_glass;
    nfd_.SofteningLengthInternal = softening_length_internal;
    WriteState.DensityKernelRad2 = b2;
    RescaleAndCoAddAcceleration(0);
    return 0;
}

/* KickSlab over one slab of cpd x cpd cells (cell_start[cpd*cpd + 1]):
 * velocities updated in place; stats[3 * cell] = mean square velocity, max
 * |v| component, max |a| component; aux_dens (optional) receives acc.w. */
extern "C" int nfrefkick_kick_slab(int cpd, const int64_t *cell_start, float *vel, float *acc,
                                   float kick1, float kick2, float *stats, float *aux_dens) {
    if (cpd <= 0 || !cell_start || !vel || !acc || !stats) return -1;
    const int64_t ncell = (int64_t)cpd * cpd;
    g.cpd = cpd;
    g.cell_start = cell_start;
    g.vel = (velstruct *)vel;
    g.acc = (accstruct *)acc;
    g.aux = aux_dens ? (shim_aux *)aux_dens : nullptr;
    g.ci = (shim_cellinfo *)stats;
    cp_.cpd = cpd;
    node_z_start = 0;
    node_z_size = cpd;
    (void)ncell;
    KickSlab(0, kick1, kick2, aux_dens != nullptr, KickCell);
    return 0;
}
