// ref_gpu_shim.cu -- TEST INFRASTRUCTURE (a checker, never the product).
//
// Builds the reference's own GPU pencil kernel, ComputeDirects
// (singlestep/Direct/PencilKernel.cu:97-188, pair kernels of
// singlestep/Direct/DirectGPUKernels.cuh), from its unmodified sources for
// sm_100a, with the reference's default GPU configuration: --use_fast_math
// (common.mk.in:31), BLOCK_ACCUM and COMPUTE_FOF_DENSITY on (configure.ac),
// NFBlockSize 64, NFRADIUS 2.  The softening is chosen with the same
// -DDIRECT* macros as the reference build.
//
// This file only supplies what GPUControl.cu and PencilTask.cu would around
// the kernel: the FLOAT / accstruct macros (GPUControl.cu:115-139), the
// interaction counter, and the launch record the kernel reads (its field
// names are those of PencilTask.cu:28-45, because the kernel reads them),
// plus one extern "C" entry that copies a SIC's arrays to the device,
// launches the kernel (repeats times) and returns the accelerations and
// the mean launch time.  The arrays are built by oracle/oracle.py in the
// reference's SIC layout.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

typedef uint64_t uint64;
#define FLOAT float
#define FLOAT3 float3
#define FLOAT4 float4
#define RSQRT rsqrtf
#define MIN fminf
#ifdef COMPUTE_FOF_DENSITY
#define accstruct FLOAT4
#else
#define accstruct FLOAT3
#endif
#define NFBlockSize 64

#include "GPUStructureOfLists.cc"

__device__ unsigned long long int DI;

#include "IncludeGPUKernels.cuh"

struct DeviceData {
    List3<FLOAT> SinkSetPositions;
    List3<FLOAT> SourceSetPositions;
    unsigned int *SinkSetIdMax;
    accstruct *SinkSetAccelerations;
    int *SinkBlockParentPencil;
    int *SourceSetStart;
    int *SourceSetCount;
    int *SinkSourceInteractionList;
    FLOAT *SinkSourceYOffset;
    FLOAT b2;
    int nfwidth;
};

#include "PencilKernel.cu"

template <class T>
static cudaError_t up(T **d, const T *h, size_t n) {
    cudaError_t e = cudaMalloc((void **)d, (n ? n : 1) * sizeof(T));
    if (e == cudaSuccess && n) e = cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

// sink_xyz: 3 x n_sink_slots floats (X | Y | Z), padded pencils;
// source_xyz: 3 x n_source floats; acc_out: n_sink_slots x (3 or 4) floats.
extern "C" int nfrefgpu_run(int nsinkblocks, int nsinkslots, const float *sink_xyz,
                            const unsigned int *sink_id_max, const int *block_parent, int nsource,
                            const float *source_xyz, int nsourcesets, const int *source_start,
                            const int *source_count, int ninteractions, const int *ilist,
                            const float *yoffset, float eps, float b2, int repeats, float *acc_out,
                            float *ms_out) {
    DeviceData d;
    memset(&d, 0, sizeof(d));
    float *sx = nullptr, *so = nullptr, *yo = nullptr;
    cudaError_t e = up(&sx, sink_xyz, (size_t)3 * nsinkslots);
    if (e == cudaSuccess) e = up(&so, source_xyz, (size_t)3 * nsource);
    if (e == cudaSuccess) e = up(&d.SinkSetIdMax, sink_id_max, (size_t)(ninteractions / 5));
    if (e == cudaSuccess) e = up(&d.SinkBlockParentPencil, block_parent, (size_t)nsinkblocks);
    if (e == cudaSuccess) e = up(&d.SourceSetStart, source_start, (size_t)nsourcesets);
    if (e == cudaSuccess) e = up(&d.SourceSetCount, source_count, (size_t)nsourcesets);
    if (e == cudaSuccess) e = up(&d.SinkSourceInteractionList, ilist, (size_t)ninteractions);
    if (e == cudaSuccess) e = up(&yo, yoffset, (size_t)ninteractions);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&d.SinkSetAccelerations,
                       (size_t)(nsinkslots ? nsinkslots : 1) * sizeof(accstruct));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    if (e == cudaSuccess) {
        d.SinkSetPositions = List3<FLOAT>{(uint64)nsinkslots, sx, sx + nsinkslots, sx + 2 * (size_t)nsinkslots};
        d.SourceSetPositions = List3<FLOAT>{(uint64)nsource, so, so + nsource, so + 2 * (size_t)nsource};
        d.SinkSourceYOffset = yo;
        d.b2 = b2;
        d.nfwidth = 5;
        // one launch to warm up, then repeats timed launches (same result)
        if (nsinkblocks > 0) ComputeDirects<<<nsinkblocks, NFBlockSize>>>(d, eps);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(t0);
        for (int r = 0; r < repeats && e == cudaSuccess; r++) {
            if (nsinkblocks > 0) ComputeDirects<<<nsinkblocks, NFBlockSize>>>(d, eps);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaEventRecord(t1);
        if (e == cudaSuccess) e = cudaEventSynchronize(t1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
        if (ms_out) *ms_out = repeats > 0 ? ms / repeats : 0.f;
        if (e == cudaSuccess && nsinkslots)
            e = cudaMemcpy(acc_out, d.SinkSetAccelerations, (size_t)nsinkslots * sizeof(accstruct),
                           cudaMemcpyDeviceToHost);
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(sx);
    cudaFree(so);
    cudaFree(yo);
    cudaFree(d.SinkSetIdMax);
    cudaFree(d.SinkBlockParentPencil);
    cudaFree(d.SourceSetStart);
    cudaFree(d.SourceSetCount);
    cudaFree(d.SinkSourceInteractionList);
    cudaFree(d.SinkSetAccelerations);
    return (int)e;
}

extern "C" int nfrefgpu_accstruct_floats() { return (int)(sizeof(accstruct) / sizeof(float)); }
