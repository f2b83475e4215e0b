// driver_plan.cpp -- a C++ consumer of the C ABI, the way abacus binds it
// (no Python): a small box laid out as abacus holds it (per-slab PosXYZ
// X | Y | Z and cellinfo, particles in (y, z) cell order), registered with
// the NearFieldDriver mirror in planner-only mode (device = -1), one SIC per
// slab planned, and DirectTotal checked against the 5x5x5 pair count
// (DirectBench.cpp:111-125), for one z-domain and for the nodes of a 2D
// z-split.  Prints "ok <pairs>" and exits 0 on success.
#include <cstdio>
#include <vector>

#include "nf_capi.h"

namespace {

constexpr int CPD = 7, R = 2;

int cell_count(int x, int y, int z) { return (x * 3 + y * 5 + z * 7) % 6; }  // 0..5, some empty

int wrap(int i) { return ((i % CPD) + CPD) % CPD; }

struct Slab {
    std::vector<float> pos;
    std::vector<nf_cellinfo> ci;
    std::vector<float> acc;
};

Slab make_slab(int x, int zs, int zn) {
    // 2D node (zn > 0): rows hold the cells zs-R .. zs+zn+R-1, startindex
    // counts the primary cells only; zn = 0: all cells, both indices equal
    Slab s;
    s.ci.assign(CPD * CPD, nf_cellinfo{0, 0, 0, 0, 0.f, 0.f, 0.f});
    std::vector<float> X, Y, Z;
    uint64_t ng = 0, np = 0;
    const int lo = zn ? zs - R : 0, hi = zn ? zs + zn + R : CPD;
    for (int y = 0; y < CPD; y++)
        for (int zz = lo; zz < hi; zz++) {
            const int z = wrap(zz);
            const int n = cell_count(x, y, z);
            const bool primary = !zn || (zz >= zs && zz < zs + zn);
            nf_cellinfo &c = s.ci[y * CPD + z];
            c.startindex_with_ghost = ng;
            c.startindex = np;
            c.count = n;
            c.active = n;
            for (int i = 0; i < n; i++) {
                X.push_back(0.01f * i);
                Y.push_back(-0.01f * i);
                Z.push_back(0.005f * i);
            }
            ng += n;
            if (primary) np += n;
        }
    s.pos = X;
    s.pos.insert(s.pos.end(), Y.begin(), Y.end());
    s.pos.insert(s.pos.end(), Z.begin(), Z.end());
    s.acc.assign(4 * (np ? np : 1), 0.f);
    return s;
}

uint64_t brute_pairs(int zs, int zn) {
    uint64_t t = 0;
    for (int x = 0; x < CPD; x++)
        for (int y = 0; y < CPD; y++)
            for (int z = 0; z < CPD; z++) {
                if (zn && wrap(z - zs) >= zn) continue;
                uint64_t m = 0;
                for (int a = -R; a <= R; a++)
                    for (int b = -R; b <= R; b++)
                        for (int c = -R; c <= R; c++) m += cell_count(wrap(x + a), wrap(y + b), wrap(z + c));
                t += (uint64_t)cell_count(x, y, z) * m;
            }
    return t;
}

int plan_total(int zs, int zn, uint64_t *total) {
    std::vector<Slab> slabs;
    int64_t n = 0;
    for (int x = 0; x < CPD; x++) {
        slabs.push_back(make_slab(x, zs, zn));
        for (int i = 0; i < CPD * CPD; i++) n += slabs.back().ci[i].count;
    }
    nf_driver_params p = {};
    p.device = -1;  // planner only
    p.cpd = CPD;
    p.np = n;
    p.near_field_radius = R;
    p.softening = NF_SOFT_PLUMMER;
    p.softening_length = 1e-3;
    p.direct_bpd = 1;
    p.mem_per_gpu_buffer_gb = 0.05;
    p.use_pinned_gpu_memory = -1;
    p.accumulation = NF_ACC_COMPENSATED;
    p.out_kind = NF_OUT_FLOAT4;
    p.node_z_start = zs;
    p.node_z_size = zn;
    nf_driver *drv = nullptr;
    if (nf_driver_create(&p, &drv) != NF_OK) {
        std::printf("create: %s\n", nf_last_error());
        return 1;
    }
    for (int x = 0; x < CPD; x++) {
        nf_slab_view v = {slabs[x].pos.data(), (uint64_t)(slabs[x].pos.size() / 3), slabs[x].ci.data(),
                          slabs[x].acc.data()};
        if (nf_driver_set_slab(drv, x, &v) != NF_OK) {
            std::printf("set_slab: %s\n", nf_last_error());
            nf_driver_destroy(drv);
            return 1;
        }
    }
    *total = 0;
    for (int x = 0; x < CPD; x++) {
        nf_sic_summary s;
        if (nf_driver_plan_sic(drv, x, 0, CPD, &s, nullptr, nullptr, nullptr) != NF_OK) {
            std::printf("plan: %s\n", nf_last_error());
            nf_driver_destroy(drv);
            return 1;
        }
        *total += s.direct_total;
    }
    nf_driver_destroy(drv);
    return 0;
}

}  // namespace

int main() {
    if (nf_abi_version() != NF_ABI_VERSION) {
        std::printf("ABI version %d, header %d\n", nf_abi_version(), NF_ABI_VERSION);
        return 1;
    }
    uint64_t one = 0, split = 0;
    if (plan_total(0, 0, &one)) return 1;
    const uint64_t want = brute_pairs(0, 0);
    if (one != want) {
        std::printf("one domain: %llu pairs planned, %llu expected\n", (unsigned long long)one,
                    (unsigned long long)want);
        return 1;
    }
    const int nodes[3][2] = {{0, 3}, {3, 2}, {5, 2}};  // z cells 0-2, 3-4, 5-6
    for (const auto &nd : nodes) {
        uint64_t t = 0;
        if (plan_total(nd[0], nd[1], &t)) return 1;
        if (t != brute_pairs(nd[0], nd[1])) {
            std::printf("node (%d, %d): %llu pairs planned, %llu expected\n", nd[0], nd[1],
                        (unsigned long long)t, (unsigned long long)brute_pairs(nd[0], nd[1]));
            return 1;
        }
        split += t;
    }
    if (split != one) {
        std::printf("nodes sum to %llu, one domain %llu\n", (unsigned long long)split,
                    (unsigned long long)one);
        return 1;
    }
    std::printf("ok %llu\n", (unsigned long long)one);
    return 0;
}
