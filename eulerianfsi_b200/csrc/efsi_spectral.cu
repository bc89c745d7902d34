// efsi_spectral.cu — direct solve of the projection's Poisson problem by fast
// diagonalisation (Lynch, Rice and Thomas, "Direct solution of partial difference
// equations by tensor product methods", Numer. Math. 6, 1964).
//
// On a uniform grid the level-0 operator of the projection (cell-area weighted -L,
// Projection.jl:106-113 for the matrix) is K = ax (Tx (x) I) + ay (I (x) Ty), with Tx,
// Ty the 1-D second-difference operators whose end rows carry the boundary kind of each
// side (Neumann: 1, Dirichlet: 3, periodic: wrap).  Each 1-D operator is diagonalised by
// a real transform, evaluated with a power-of-two complex FFT in shared memory:
//   Neumann-Neumann      DCT-II (Makhoul, IEEE Trans. ASSP 28, 1980: even/odd reorder,
//                        one complex FFT of length n, a post-twiddle)   mu = 2 - 2 cos(pi k / n)
//   Dirichlet-Dirichlet  DCT-II of (-1)^i x (DST-II with reversed modes) mu = 2 + 2 cos(pi k / n)
//   Neumann-Dirichlet    odd extension about the Dirichlet face, DCT-II of length 2n, odd modes
//                        (DCT-IV)                                        mu = 2 - 2 cos(pi (2k+1) / 2n)
//   Dirichlet-Neumann    the same on the reversed index
//   periodic             Hartley transform (Re F - Im F)                  mu = 2 - 2 cos(2 pi k / n)
// so K^-1 = Fx^-1 Fy^-1 diag(1 / (ax mu_x + ay mu_y)) Fy Fx (the zero mode of a singular
// operator is dropped: the zero-mean solution).  The solve is used as the exact inverse
// of a Richardson iteration x += K^-1 (b - K x) judged by the FP64 residual, so the
// projection's relative tolerance keeps its meaning; one iteration reaches about 1e-13.
//
// Data flow of one iteration (four launches, the arrays stay L2-resident at 1024^2); the
// solve's init has stored r = (b - mean) - K x0 and decided on it:
//   A  rows j: x transform of r, modes written transposed (T[j + k Ny]);
//   B  modes k: y transform, division by the eigenvalue, inverse y transform, written
//      transposed back (T2[k + j Nx]);
//   C  rows j: inverse x transform, x += e;
//   R  cells: r = (b - mean) - K x (FP64, stored), |r|^2 decides convergence.
// A converged solve therefore ends after its R, with no transform spent on the test.
#include "efsi_solvers.cuh"

namespace efsi {

namespace {

constexpr int kSpecThreads = 512;  // with at most 64 registers: two blocks (the shared-memory limit) fill an SM

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ int brev(int i, int logL) { return (int)(__brev((unsigned)i) >> (32 - logL)); }
// Padded shared-memory slot of FFT element i (one spare element per 32, so that the
// bit-reversed scatters and the butterflies of a warp spread over the banks).
__device__ __forceinline__ int pad(int i) { return i + (i >> 5); }

// Slot of twiddle t in shared memory: the low three bits are XORed with a fold of the
// higher bits, so that the power-of-two strides of the butterfly passes (t = j ts over
// consecutive j) spread over the eight 16-byte bank groups; a permutation of [0, L/2).
__device__ __forceinline__ int twz(int t) {
    const int x = t >> 3;
    return t ^ ((x ^ (x >> 3) ^ (x >> 6) ^ (x >> 9)) & 7);
}
// Row stride (doubles) of the transposed-mode tiles: rows padded by 8 doubles, so that
// the column-wise reads of four rows fall on different banks.
__device__ __forceinline__ int tile_row(int n) { return n + 8; }

// Shared-memory layout of one block: the L/2 twiddles (slots twz(t)), then R FFT rows of
// spectral_row(L) padded elements (R rows are transformed at once, with the same
// barriers as one).
__device__ __forceinline__ double2* fft_rows(unsigned char* smem, const SpecDir& d) {
    return reinterpret_cast<double2*>(smem) + d.L / 2;
}
__device__ __forceinline__ void load_twiddles(unsigned char* smem, const SpecDir& d) {
    double2* tw = reinterpret_cast<double2*>(smem);
    for (int t = threadIdx.x; t < d.L / 2; t += blockDim.x) tw[twz(t)] = __ldg(d.w + t);
}

// W consecutive radix-2 decimation-in-time stages s0 + 1 .. s0 + W (stage s pairs
// elements 2^(s-1) apart, twiddle exp(-2 pi i j / 2^s) for the pair's offset j within its
// half-block) done in registers on groups of 2^W elements {b + j + m 2^s0}: one shared-
// memory read and write of each element and one barrier per W stages instead of per
// stage.  With the padded layout a warp's 16-byte accesses of one m fall on distinct
// bank groups for every distance (consecutive j, or contiguous runs of 8 for s0 = 0).
template <int W>
__device__ __forceinline__ void fft_pass(double2* a, const double2* tw, int L, int logL, int stride, int s0, int R) {
    constexpr int M = 1 << W;
    const int h = 1 << s0, lg = logL - W, G = L >> W;  // G groups per row
    for (int q = threadIdx.x; q < R * G; q += blockDim.x) {
        const int r = q >> lg, g = q & (G - 1);
        const int j = g & (h - 1), b = (g >> s0) << (s0 + W);
        double2* row = a + (size_t)r * stride;
        double2 v[M];
#pragma unroll
        for (int m = 0; m < M; ++m) v[m] = row[pad(b + j + m * h)];
#pragma unroll
        for (int t = 0; t < W; ++t) {
            const int hs = 1 << t, ts = L >> (s0 + t + 1);
#pragma unroll
            for (int m = 0; m < M; ++m) {
                if (m & hs) continue;  // m is the lower element of the pair (m, m + hs)
                const double2 x = cmul(tw[twz((j + (m & (hs - 1)) * h) * ts)], v[m + hs]), u = v[m];
                v[m] = make_double2(u.x + x.x, u.y + x.y);
                v[m + hs] = make_double2(u.x - x.x, u.y - x.y);
            }
        }
#pragma unroll
        for (int m = 0; m < M; ++m) row[pad(b + j + m * h)] = v[m];
    }
    __syncthreads();
}

// In-place FFT (forward sign) of R rows a[r * stride + pad(.)] whose inputs are stored in
// bit-reversed order, as radix-8 register passes (the last pass radix-4 or radix-2 when
// log2 L is not a multiple of 3); ends with a barrier.
__device__ void fft_smem(double2* a, const double2* tw, const SpecDir& d, int R) {
    const int L = d.L, stride = spectral_row(L);
    for (int s0 = 0; s0 < d.logL;) {
        const int w = d.logL - s0;
        if (w >= 3) { fft_pass<3>(a, tw, L, d.logL, stride, s0, R); s0 += 3; }
        else if (w == 2) { fft_pass<2>(a, tw, L, d.logL, stride, s0, R); s0 += 2; }
        else { fft_pass<1>(a, tw, L, d.logL, stride, s0, R); s0 += 1; }
    }
}

// Position of input e (0 <= e < L) in the bit-reversed FFT input of the Makhoul DCT-II:
// v_m = x_2m, v_(L-1-m) = x_(2m+1).
__device__ __forceinline__ int dct_slot(int e, const SpecDir& d) {
    const int p = (e & 1) ? d.L - 1 - (e >> 1) : (e >> 1);
    return pad(brev(p, d.logL));
}

// Forward transform, scatter of input value x at index i (0 <= i < n) into one row.
__device__ __forceinline__ void fwd_put(double2* a, const SpecDir& d, int i, double x) {
    switch (d.kind) {
    case SPEC_NN: a[dct_slot(i, d)] = make_double2(x, 0.0); break;
    case SPEC_DD: a[dct_slot(i, d)] = make_double2((i & 1) ? -x : x, 0.0); break;
    case SPEC_ND:
        a[dct_slot(i, d)] = make_double2(x, 0.0);
        a[dct_slot(d.L - 1 - i, d)] = make_double2(-x, 0.0);
        break;
    case SPEC_DN: {
        const int m = d.n - 1 - i;
        a[dct_slot(m, d)] = make_double2(x, 0.0);
        a[dct_slot(d.L - 1 - m, d)] = make_double2(-x, 0.0);
        break;
    }
    default: a[pad(brev(i, d.logL))] = make_double2(x, 0.0); break;  // SPEC_P
    }
}
// Forward transform, mode k (0 <= k < n) of one row after the FFT.
__device__ __forceinline__ double fwd_get(const double2* a, const SpecDir& d, int k) {
    if (d.kind == SPEC_P) {
        const double2 v = a[pad(k)];
        return v.x - v.y;
    }
    const int kk = (d.kind == SPEC_ND || d.kind == SPEC_DN) ? 2 * k + 1 : k;
    const double2 m = __ldg(d.mk + kk), v = a[pad(kk)];
    return m.x * v.x - m.y * v.y;  // Re(exp(-i pi kk / 2L) V_kk)
}
// Inverse transform, FFT input at index k (0 <= k < L) of one row from the modes X(.)
// (0 <= . < n): the DCT-II inverse of Makhoul, conj(V_k) = exp(-i pi k / 2L) (X_k + i
// X_(L-k)), X_L = 0, with X the odd-mode embedding for ND / DN; the Hartley transform for
// periodic.
template <class G>
__device__ __forceinline__ void inv_put(double2* a, const SpecDir& d, int k, const G& X) {
    double2 c;
    if (d.kind == SPEC_P) {
        c = make_double2(X(k), 0.0);
    } else {
        double xk, xnk;
        if (d.kind == SPEC_ND || d.kind == SPEC_DN) {
            if (k & 1) { xk = X((k - 1) >> 1); xnk = X((d.L - k - 1) >> 1); }
            else { xk = 0.0; xnk = 0.0; }
        } else {
            xk = X(k);
            xnk = k == 0 ? 0.0 : X(d.L - k);
        }
        const double2 m = __ldg(d.mk + k);
        c = make_double2(m.x * xk - m.y * xnk, m.x * xnk + m.y * xk);
    }
    a[pad(brev(k, d.logL))] = c;
}
// Inverse transform, output value at index i (0 <= i < n) of one row after the FFT.
__device__ __forceinline__ double inv_get(const double2* a, const SpecDir& d, int i) {
    if (d.kind == SPEC_P) {  // 1 / n and 1 / L are exact (powers of two)
        const double2 v = a[pad(i)];
        return (v.x - v.y) * d.inv_n;
    }
    const int e = d.kind == SPEC_DN ? d.n - 1 - i : i;
    const int p = (e & 1) ? d.L - 1 - (e >> 1) : (e >> 1);
    const double v = a[pad(p)].x * d.inv_L;
    return (d.kind == SPEC_DD && (i & 1)) ? -v : v;
}

// K x at cell (i, j) of level 0 (the weighted operator with its boundary factors).
__device__ __forceinline__ double apply_K(const MGLevel& L, int px, int py, const double* x, int i, int j) {
    const int nx = L.nx, ny = L.ny;
    const size_t k = cidx(i, j, nx);
    double d = 0.0, off = 0.0;
    if (i > 0) { d += L.ax; off += L.ax * x[k - 1]; }
    else if (px) { d += L.ax; off += L.ax * x[k + nx - 1]; }
    else d += L.ax * L.cl[j];
    if (i < nx - 1) { d += L.ax; off += L.ax * x[k + 1]; }
    else if (px) { d += L.ax; off += L.ax * x[k - (nx - 1)]; }
    else d += L.ax * L.cr[j];
    if (j > 0) { d += L.ay; off += L.ay * x[k - nx]; }
    else if (py) { d += L.ay; off += L.ay * x[k + (size_t)(ny - 1) * nx]; }
    else d += L.ay * L.cb[i];
    if (j < ny - 1) { d += L.ay; off += L.ay * x[k + nx]; }
    else if (py) { d += L.ay; off += L.ay * x[k - (size_t)(ny - 1) * nx]; }
    else d += L.ay * L.ct[i];
    return d * x[k] - off;
}

// A: x transform of the residual rows j0 .. j0 + R - 1 (transformed together); the
// modes go to the tile and from there transposed to T.
__global__ void __launch_bounds__(kSpecThreads, 2) k_spec_a(Spectral sp, int nx, int ny, const double* __restrict__ r,
                                                        double* __restrict__ T, const CGScal* cg) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (cg->done) return;
    const SpecDir& d = sp.dx;
    const double2* tw = reinterpret_cast<const double2*>(smem);
    double2* a = fft_rows(smem, d);
    const int stride = spectral_row(d.L);
    const int j0 = blockIdx.x * sp.rows_a, R = sp.rows_a;  // R divides ny
    double* tile = reinterpret_cast<double*>(a + (size_t)sp.rows_a * stride);
    load_twiddles(smem, d);
    for (int q = threadIdx.x; q < R * nx; q += blockDim.x) {
        const int rr = q >> d.logn, i = q & (nx - 1);
        fwd_put(a + (size_t)rr * stride, d, i, __ldg(r + cidx(i, j0 + rr, nx)));
    }
    __syncthreads();
    fft_smem(a, tw, d, R);
    for (int q = threadIdx.x; q < R * nx; q += blockDim.x) {
        const int rr = q >> d.logn, k = q & (nx - 1);
        tile[rr * tile_row(nx) + k] = fwd_get(a + (size_t)rr * stride, d, k);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < R * nx; q += blockDim.x) {
        const int k = q >> sp.lg_a, rr = q & (R - 1);
        T[(size_t)(j0 + rr) + (size_t)k * ny] = tile[rr * tile_row(nx) + k];
    }
}

// B: y transform of modes k0 .. k0 + R - 1 (together), division by the eigenvalue,
// inverse y transform, written transposed to T2.
__global__ void __launch_bounds__(kSpecThreads, 2) k_spec_b(Spectral sp, double ax, double ay,
                                                        const double* __restrict__ T, double* __restrict__ T2,
                                                        const CGScal* cg) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (cg->done) return;
    const SpecDir& dx = sp.dx;
    const SpecDir& d = sp.dy;
    const double2* tw = reinterpret_cast<const double2*>(smem);
    double2* a = fft_rows(smem, d);
    const int stride = spectral_row(d.L);
    const int nx = dx.n, ny = d.n, k0 = blockIdx.x * sp.rows_b, R = sp.rows_b;  // R divides nx
    double* tile = reinterpret_cast<double*>(a + (size_t)sp.rows_b * stride);
    load_twiddles(smem, d);
    for (int q = threadIdx.x; q < R * ny; q += blockDim.x) {
        const int r = q >> d.logn, l = q & (ny - 1);
        fwd_put(a + (size_t)r * stride, d, l, T[(size_t)(k0 + r) * ny + l]);
    }
    __syncthreads();
    fft_smem(a, tw, d, R);
    for (int q = threadIdx.x; q < R * ny; q += blockDim.x) {
        const int r = q >> d.logn, l = q & (ny - 1);
        const double lam = ax * __ldg(dx.mu + k0 + r) + ay * __ldg(d.mu + l);
        tile[r * tile_row(ny) + l] = lam > 0.0 ? fwd_get(a + (size_t)r * stride, d, l) / lam : 0.0;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < R * d.L; q += blockDim.x) {
        const int r = q >> d.logL, kk = q & (d.L - 1);
        const double* row = tile + (size_t)r * tile_row(ny);
        inv_put(a + (size_t)r * stride, d, kk, [&](int m) { return row[m]; });
    }
    __syncthreads();
    fft_smem(a, tw, d, R);
    for (int q = threadIdx.x; q < R * ny; q += blockDim.x) {
        const int r = q >> d.logn, l = q & (ny - 1);
        tile[r * tile_row(ny) + l] = inv_get(a + (size_t)r * stride, d, l);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < R * ny; q += blockDim.x) {
        const int l = q >> sp.lg_b, r = q & (R - 1);
        T2[(size_t)(k0 + r) + (size_t)l * nx] = tile[r * tile_row(ny) + l];
    }
}

// C: inverse x transform of rows j0 .. j0 + R - 1 (together), x += e; the iteration count.
__global__ void __launch_bounds__(kSpecThreads, 2) k_spec_c(Spectral sp, const double* __restrict__ T2, double* x,
                                                        CGScal* cg, int* iters_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (cg->done) return;
    const SpecDir& d = sp.dx;
    const double2* tw = reinterpret_cast<const double2*>(smem);
    double2* a = fft_rows(smem, d);
    const int stride = spectral_row(d.L);
    const int nx = d.n, j0 = blockIdx.x * sp.rows_c, R = sp.rows_c;  // R divides ny
    load_twiddles(smem, d);
    for (int q = threadIdx.x; q < R * d.L; q += blockDim.x) {
        const int r = q >> d.logL, kk = q & (d.L - 1);
        const double* row = T2 + (size_t)(j0 + r) * nx;
        inv_put(a + (size_t)r * stride, d, kk, [&](int m) { return __ldg(row + m); });
    }
    __syncthreads();
    fft_smem(a, tw, d, R);
    for (int q = threadIdx.x; q < R * nx; q += blockDim.x) {
        const int r = q >> d.logn, i = q & (nx - 1);
        x[cidx(i, j0 + r, nx)] += inv_get(a + (size_t)r * stride, d, i);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cg->iter += 1;
        if (iters_out) *iters_out = cg->iter;
    }
}

// R: after a pass, r = (b - mean) - K x (stored for the next pass's transform) and its
// squared norm over the grid; the convergence decision of the Richardson iteration.
__global__ void __launch_bounds__(kSpecThreads, 2) k_spec_r(MGLevel L0, int logn, int px, int py,
                                                        const double* __restrict__ b, const double* __restrict__ x,
                                                        double* __restrict__ r, const ProjScal* ps, CGScal* cg,
                                                        RedSlot rs, int* iters_out, cudaGraphConditionalHandle cond) {
    __shared__ double sh[32];
    if (cg->done) return;
    const int nx = L0.nx;
    const size_t nc = (size_t)nx * L0.ny;
    const double bmean = ps->v[10];
    double acc[1] = {0.0};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nc; q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q & (size_t)(nx - 1)), j = (int)(q >> logn);
        const size_t k = cidx(i, j, nx);
        const double v = (b[k] - bmean) - apply_K(L0, px, py, x, i, j);
        r[k] = v;
        acc[0] += v * v;
    }
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0) {
        // With the exact inverse a pass leaves only the rounding of K x and of the
        // transforms (about eps |K| |x|); a pass that does not halve the residual is at
        // that floor, which no further pass lowers: accepted as converged (the
        // projection's true-residual test still judges it against its own tolerance).
        const bool stalled = tot[0] > 0.25 * cg->rr;
        cg->rr = tot[0];
        if (tot[0] <= cg->tol2 || (stalled && isfinite(tot[0]))) { cg->conv = 1; cg->done = 1; }
        else if (cg->iter >= cg->maxiter || !isfinite(tot[0])) cg->done = 1;
        if (iters_out) *iters_out = cg->iter;
        set_loop(cond, !cg->done);
    }
}

}  // namespace

cudaError_t spectral_configure(const Spectral& sp) {
    if (!sp.on) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_spec_a, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp.smem_a);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_spec_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp.smem_b);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_spec_c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp.smem_c);
    return e;
}

void proj_spectral_iter(const Params& P, const Projection& pj, CGScal* cg, const ProjScal* ps, const RedSlot& rs,
                        int* iters_out, cudaGraphConditionalHandle cond, cudaStream_t s) {
    const Spectral& sp = pj.sp;
    const MGLevel& L = pj.lev[0];
    const int ga = (L.ny + sp.rows_a - 1) / sp.rows_a, gb = (L.nx + sp.rows_b - 1) / sp.rows_b;
    const int gc = (L.ny + sp.rows_c - 1) / sp.rows_c;
    // r = pj.r[0] (the residual, from the solve's init or the previous pass's R),
    // T = pj.z (modes, y contiguous), T2 = pj.w (modes, x contiguous)
    k_spec_a<<<ga, kSpecThreads, sp.smem_a, s>>>(sp, L.nx, L.ny, pj.r[0], pj.z, cg);
    k_spec_b<<<gb, kSpecThreads, sp.smem_b, s>>>(sp, L.ax, L.ay, pj.z, pj.w, cg);
    k_spec_c<<<gc, kSpecThreads, sp.smem_c, s>>>(sp, pj.w, pj.x, cg, iters_out);
    const size_t nc = (size_t)L.nx * L.ny;
    // one persistent wave (two 512-thread blocks per SM at 64 registers)
    const int gr = (int)std::min<size_t>((nc + kSpecThreads - 1) / kSpecThreads, (size_t)std::max(P.nsm, 1) * 2);
    k_spec_r<<<gr, kSpecThreads, 0, s>>>(L, sp.dx.logn, P.g.px, P.g.py, pj.b, pj.x, pj.r[0], ps, cg, rs, iters_out,
                                         cond);
}

}  // namespace efsi
