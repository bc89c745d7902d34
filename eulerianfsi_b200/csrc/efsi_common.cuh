// efsi_common.cuh — device-side parameters, indexing, boundary data access and
// deterministic block reductions shared by every kernel of the IMEX step.
//
// Layout in HBM (all FP64 unless a precision-form buffer says otherwise), the same
// column-major order as the Julia matrices so that host<->device copies are flat:
//   U  (Nx+1) x Ny   idx = i + j*(Nx+1)
//   V  Nx x (Ny+1)   idx = i + j*Nx
//   cell Nx x Ny     idx = i + j*Nx
// The device step assumes uniform spacing (hx = Lx/Nx, hy = Ly/Ny); for uniform
// MeshMetrics every dx_f/dx_c/dy_f/dy_c entry equals hx/hy, every interior
// interpolation weight is 1/2 and every corner distance is h/2
// (MeshGeneration.jl:237-335), which is what the stencils below encode.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/efsi.h"

namespace efsi {

// ---- boundary data ------------------------------------------------------------------
struct SideD {
    int type;                // EFSI_BC_*
    const double* val;       // device array (Dirichlet / Neumann / mixed-Dirichlet / backflow)
    const double* neu;       // mixed Neumann data
    const uint8_t* mask;     // mixed Dirichlet mask
};
struct BCD {
    SideD s[4];  // left, right, bottom, top
};
enum { LEFT = 0, RIGHT = 1, BOTTOM = 2, TOP = 3 };

__device__ __forceinline__ double bval(const SideD& s, int k) { return s.val ? s.val[k] : 0.0; }
__device__ __forceinline__ double bneu(const SideD& s, int k) { return s.neu ? s.neu[k] : 0.0; }
__device__ __forceinline__ bool bdir(const SideD& s, int k) {
    return s.type == EFSI_BC_DIRICHLET || (s.type == EFSI_BC_MIXED && s.mask && s.mask[k]);
}

struct GridD {
    int Nx, Ny;
    int px, py;
    double hx, hy, ihx, ihy;
    double Lx, Ly;
};

// Everything a kernel needs, passed by value (kernel parameter space).
struct Params {
    GridD g;
    BCD bu, bv, bq, bphi, bc, bsxx, bsyy, bsxy;
    efsi_models md;
    efsi_numerics nu;
    double psi_bc[4];  // ACDI: psi of the scalar Dirichlet phase data per side (PhaseFieldMethods.jl:509-516)
    int nsm;           // multiprocessors of the device (persistent launch grids)
};

// Grid of a persistent (grid-stride over tiles) launch: at most `per_sm` blocks per SM.
inline int persistent_grid(int ntiles, int nsm, int per_sm) {
    int cap = (nsm > 0 ? nsm : 148) * per_sm;
    return ntiles < 1 ? 1 : (ntiles < cap ? ntiles : cap);
}

// ---- device error flags ---------------------------------------------------------------
// First error wins; the host maps `code` to an EFSI_* status and a message.
enum DevErr : int {
    DE_NONE = 0,
    DE_NONFINITE_STATE = 1,     // ArgumentError, TimeIntegrationIMEX.jl:517-521
    DE_STAGE1_CONSTRAINT = 2,   // ArgumentError, TimeIntegrationIMEX.jl:1121
    DE_INCOMPATIBLE = 3,        // ArgumentError, Projection.jl:213
    DE_PROJ_RESIDUAL = 4,       // ErrorException, Projection.jl:281
    DE_PROJ_CONSTRAINT = 5,     // ErrorException, Projection.jl:293
    DE_NON_SPD = 6,             // DomainError, StructureTensor.jl:491
    DE_NEUMANN_INFLOW = 7,      // ArgumentError, InterfaceTransport.jl:110 / StructureTensor.jl:218 / ResourceTransport.jl:136
    DE_BAD_VISCOSITY = 8,       // ArgumentError, TransportConstitutive.jl:66-71
    DE_BAD_DIFFUSIVITY = 9,     // ArgumentError, TransportConstitutive.jl:66-71
    DE_NONFINITE_SINK = 10,     // ArgumentError, TransportConstitutive.jl:295
    DE_LINEAR_NOCONV = 11,      // ErrorException, TimeIntegrationIMEX.jl:637
    DE_PHASE_NEUMANN = 12,      // ArgumentError, PhaseFieldMethods.jl:179
    DE_NONFINITE_INPUT = 13,    // ArgumentError on operator inputs
};

struct DevStatus {
    int code;
    int where;      // stage or field index
    int i, j;       // cell / face of the first failure
    double value;   // offending value
};

__device__ __forceinline__ void raise_err(DevStatus* st, int code, int where, int i, int j, double v) {
    if (atomicCAS(&st->code, 0, code) == 0) {
        st->where = where;
        st->i = i;
        st->j = j;
        st->value = v;
    }
}

// Time-step dependent coefficient read from device memory (dt * coef), so that a
// captured CUDA graph of the step is valid for every dt.
struct DtCoef {
    const double* dt;
    double coef;
    __device__ __forceinline__ double value() const { return *dt * coef; }
};

// Loop control of a CUDA-graph WHILE node: 0 when the kernel runs outside a graph.
__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle h, bool keep_going) {
    if (h) cudaGraphSetConditional(h, keep_going ? 1u : 0u);
}

// ---- indexing ------------------------------------------------------------------------------
__device__ __forceinline__ int wrapi(int k, int n) { return k < 0 ? k + n : (k >= n ? k - n : k); }
// any k (tile halos may reach several periods past a small level)
__device__ __forceinline__ int wrapm(int k, int n) { int m = k % n; return m < 0 ? m + n : m; }
__device__ __forceinline__ size_t cidx(int i, int j, int Nx) { return (size_t)i + (size_t)j * Nx; }
__device__ __forceinline__ size_t uidx(int i, int j, int Nx) { return (size_t)i + (size_t)j * (Nx + 1); }
__device__ __forceinline__ size_t vidx(int i, int j, int Nx) { return (size_t)i + (size_t)j * Nx; }

__device__ __forceinline__ double clamp01(double x) { return fmin(fmax(x, 0.0), 1.0); }

// ---- deterministic reductions ----------------------------------------------------------------
// Block-level sum of NV values (blockDim.x*blockDim.y threads, multiple of 32).
template <int NV, int M>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (&sh)[M]) {
    static_assert(M >= 32 * NV, "block reduction scratch needs 32 doubles per reduced value");
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    const int warp = tid >> 5, lane = tid & 31, nw = nthr >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? sh[k * 32 + lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
    __syncthreads();
}

template <int NV, int M>
__device__ __forceinline__ void block_max(double (&v)[NV], double (&sh)[M]) {
    static_assert(M >= 32 * NV, "block reduction scratch needs 32 doubles per reduced value");
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_down_sync(0xffffffffu, v[k], o));
    const int warp = tid >> 5, lane = tid & 31, nw = nthr >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? sh[k * 32 + lane] : -1.0e308;
            for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
            v[k] = x;
        }
    }
    __syncthreads();
}

// Grid-level reduction finished by the last block to arrive (fixed summation
// order, hence deterministic for a fixed launch shape).  Each block passes its
// block-reduced values (valid in thread 0); the last block receives the grid
// totals in `tot` (valid in thread 0) and returns true.
struct RedSlot {
    double* part;        // [NV][maxBlocks]
    unsigned* ticket;    // zero-initialised counter
    int maxBlocks;
};

template <int NV, bool MAXOP = false, int M>
__device__ bool grid_reduce(double (&v)[NV], const RedSlot& rs, double (&tot)[NV], double (&sh)[M]) {
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
    const int nb = gridDim.x * gridDim.y;
    const int bid = blockIdx.x + blockIdx.y * gridDim.x;
    if (MAXOP) block_max<NV>(v, sh);
    else block_sum<NV>(v, sh);
    __shared__ bool last;
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) rs.part[(size_t)k * rs.maxBlocks + bid] = v[k];
        __threadfence();
        unsigned t = atomicAdd(rs.ticket, 1u);
        last = (t == (unsigned)nb - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // The last block reads nb x NV partials from L2.  Each round issues U x NV
    // independent loads before the first add, so a thread waits about
    // nb / (nthr * U) load latencies, not nb / nthr * NV of them.
    constexpr int U = NV >= 8 ? 1 : (NV >= 4 ? 2 : 8 / NV);
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = MAXOP ? -1.0e308 : 0.0;
    int b = tid;
    for (; b + (U - 1) * nthr < nb; b += U * nthr) {
        double x[U][NV];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k = 0; k < NV; ++k) x[u][k] = __ldcg(&rs.part[(size_t)k * rs.maxBlocks + b + u * nthr]);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k = 0; k < NV; ++k) acc[k] = MAXOP ? fmax(acc[k], x[u][k]) : acc[k] + x[u][k];
    }
    for (; b < nb; b += nthr) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = __ldcg(&rs.part[(size_t)k * rs.maxBlocks + b]);
            acc[k] = MAXOP ? fmax(acc[k], x) : acc[k] + x;
        }
    }
    if (MAXOP) block_max<NV>(acc, sh);
    else block_sum<NV>(acc, sh);
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) tot[k] = acc[k];
        *rs.ticket = 0u;
    }
    return true;
}

}  // namespace efsi
