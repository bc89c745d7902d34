// efsi_diag.cu — the cavity drivers' per-step diagnostics on the device-resident
// state (scripts/benchmarks/run_sugiyama_lid_driven_cavity.jl:484-828,
// scripts/benchmarks/BenchmarkUtilities.jl:62-87), so that a time loop reads a few
// hundred bytes instead of downloading the state.  Two reduction passes: the first
// gives the phase mass and moments (hence the centroid), the phase bounds, the flow
// and tensor-region statistics; the second the covariance and boundary Fourier
// modes about that centroid.  Block partials are reduced in a fixed order.
#include "efsi_diag.cuh"

namespace efsi {

namespace {
constexpr int DX = 32, DY = 8;
constexpr double kPi = 3.14159265358979323846;

// Face gradient of phi on the left face of cell (i, j) (scalar_gradient with the
// phi boundaries, Operators.jl:189-356); i == Nx gives the right wall face.
__device__ __forceinline__ double phi_grad_x(const Params& P, const double* phi, int i, int j) {
    const int Nx = P.g.Nx;
    auto f = [&](int a) { return phi[cidx(a, j, Nx)]; };
    if (i > 0 && i < Nx) return (f(i) - f(i - 1)) / P.g.hx;
    if (P.g.px) return (f(0) - f(Nx - 1)) / P.g.hx;
    const SideD& s = P.bphi.s[i == 0 ? LEFT : RIGHT];
    const double in = f(i == 0 ? 0 : Nx - 1), dist = P.g.hx / 2.0, sgn = i == 0 ? -1.0 : 1.0;
    if (bdir(s, j)) return sgn < 0 ? in / dist - bval(s, j) / dist : bval(s, j) / dist - in / dist;
    if (s.type == EFSI_BC_NEUMANN) return sgn * bval(s, j);
    if (s.type == EFSI_BC_MIXED) return sgn * bneu(s, j);
    return 0.0;
}
__device__ __forceinline__ double phi_grad_y(const Params& P, const double* phi, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    auto f = [&](int b) { return phi[cidx(i, b, Nx)]; };
    if (j > 0 && j < Ny) return (f(j) - f(j - 1)) / P.g.hy;
    if (P.g.py) return (f(0) - f(Ny - 1)) / P.g.hy;
    const SideD& s = P.bphi.s[j == 0 ? BOTTOM : TOP];
    const double in = f(j == 0 ? 0 : Ny - 1), dist = P.g.hy / 2.0, sgn = j == 0 ? -1.0 : 1.0;
    if (bdir(s, i)) return sgn < 0 ? in / dist - bval(s, i) / dist : bval(s, i) / dist - in / dist;
    if (s.type == EFSI_BC_NEUMANN) return sgn * bval(s, i);
    if (s.type == EFSI_BC_MIXED) return sgn * bneu(s, i);
    return 0.0;
}

__device__ __forceinline__ bool in_region(int r, double p, const efsi_diag_config& c) {
    switch (r) {
        case 0: return true;
        case 1: return p >= c.sigma_core_cutoff;
        case 2: return c.sigma_interface_cutoff < p && p < c.sigma_core_cutoff;
        default: return c.sigma_safety_cutoff < p && p <= c.sigma_interface_cutoff;
    }
}

__global__ void __launch_bounds__(DX * DY) k_diag1(Params P, efsi_diag_config cfg, const double* __restrict__ U,
                                                   const double* __restrict__ V, const double* __restrict__ phi,
                                                   const double* __restrict__ sxx, const double* __restrict__ syy,
                                                   const double* __restrict__ sxy, RedSlot rs_sum, RedSlot rs_max,
                                                   double* tot) {
    __shared__ double sh[kDiagSums > kDiagMaxes ? kDiagSums * 32 : kDiagMaxes * 32];
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double area = P.g.hx * P.g.hy;
    const int ntx = (Nx + DX - 1) / DX, nt = ntx * ((Ny + DY - 1) / DY);
    double S[kDiagSums], M[kDiagMaxes];
#pragma unroll
    for (int k = 0; k < kDiagSums; ++k) S[k] = 0.0;
#pragma unroll
    for (int k = 0; k < kDiagMaxes; ++k) M[k] = -1.0e308;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i = (t % ntx) * DX + threadIdx.x, j = (t / ntx) * DY + threadIdx.y;
        if (i >= Nx || j >= Ny) continue;
        const size_t k = cidx(i, j, Nx);
        const double p = phi[k];
        const double xp = (i + 0.5) * (P.g.Lx / Nx), yp = (j + 0.5) * (P.g.Ly / Ny);
        const double w = p * area;
        S[0] += w;
        S[1] += xp * w;
        S[2] += yp * w;
        const double pb = fmin(fmax(p, 0.0), 1.0);
        const double gx = 0.5 * phi_grad_x(P, phi, i, j) + 0.5 * phi_grad_x(P, phi, i + 1, j);
        const double gy = 0.5 * phi_grad_y(P, phi, i, j) + 0.5 * phi_grad_y(P, phi, i, j + 1);
        S[3] += area * hypot(gx, gy);
        S[4] += area * 4.0 * pb * (1.0 - pb);
        const double uL = U[uidx(i, j, Nx)], uR = U[uidx(i + 1, j, Nx)];
        const double vB = V[vidx(i, j, Nx)], vT = V[vidx(i, j + 1, Nx)];
        const double u = 0.5 * (uL + uR), v = 0.5 * (vB + vT);
        const double s2 = u * u + v * v;
        S[5] += 0.5 * cfg.density * s2 * area;
        const double div = (uR - uL) / P.g.hx + (vT - vB) / P.g.hy;
        S[6] += area * div * div;
        S[7] += area;
        S[8] += (p < 0.0 || p > 1.0) ? 1.0 : 0.0;
        M[0] = fmax(M[0], -p);
        M[1] = fmax(M[1], p);
        M[2] = fmax(M[2], sqrt(s2));
        M[3] = fmax(M[3], fabs(div));
        M[4] = fmax(M[4], fabs(uL));
        if (i == Nx - 1) M[4] = fmax(M[4], fabs(uR));
        M[5] = fmax(M[5], fabs(vB));
        if (j == Ny - 1) M[5] = fmax(M[5], fabs(vT));
        // tensor_cell_diagnostics_2d (BenchmarkUtilities.jl:62-87)
        const double xx = sxx[k], yy = syy[k], xy = sxy[k];
        const double det = xx * yy - xy * xy, tr = xx + yy, gap = hypot(xx - yy, 2.0 * xy);
        const double lmin = 0.5 * (tr - gap), lmax = 0.5 * (tr + gap), de = fabs(det - 1.0);
        const double st = fabs(p * cfg.elastic_modulus) *
                          sqrt((xx - 1.0) * (xx - 1.0) + (yy - 1.0) * (yy - 1.0) + 2.0 * xy * xy);
        const bool nonspd = !(isfinite(lmin) && lmin > 0.0);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (!in_region(r, p, cfg)) continue;
            S[9 + 5 * r + 0] += 1.0;
            S[9 + 5 * r + 1] += area;
            S[9 + 5 * r + 2] += area * de;
            S[9 + 5 * r + 3] += area * st;
            S[9 + 5 * r + 4] += nonspd ? 1.0 : 0.0;
            M[6 + 6 * r + 0] = fmax(M[6 + 6 * r + 0], -det);
            M[6 + 6 * r + 1] = fmax(M[6 + 6 * r + 1], det);
            M[6 + 6 * r + 2] = fmax(M[6 + 6 * r + 2], de);
            M[6 + 6 * r + 3] = fmax(M[6 + 6 * r + 3], -lmin);
            M[6 + 6 * r + 4] = fmax(M[6 + 6 * r + 4], lmax);
            M[6 + 6 * r + 5] = fmax(M[6 + 6 * r + 5], st);
        }
    }
    double ts[kDiagSums], tm[kDiagMaxes];
    if (grid_reduce<kDiagSums>(S, rs_sum, ts, sh) && threadIdx.x == 0 && threadIdx.y == 0)
        for (int k = 0; k < kDiagSums; ++k) tot[k] = ts[k];
    if (grid_reduce<kDiagMaxes, true>(M, rs_max, tm, sh) && threadIdx.x == 0 && threadIdx.y == 0)
        for (int k = 0; k < kDiagMaxes; ++k) tot[kDiagSums + k] = tm[k];
}

__global__ void __launch_bounds__(DX * DY) k_diag2(Params P, efsi_diag_config cfg, const double* __restrict__ phi,
                                                   RedSlot rs, double* tot) {
    __shared__ double sh[kDiagSums2 * 32];
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double area = P.g.hx * P.g.hy;
    const double mass = tot[0], xc = tot[1] / mass, yc = tot[2] / mass;
    const int ntx = (Nx + DX - 1) / DX, nt = ntx * ((Ny + DY - 1) / DY);
    double S[kDiagSums2];
#pragma unroll
    for (int k = 0; k < kDiagSums2; ++k) S[k] = 0.0;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int i = (t % ntx) * DX + threadIdx.x, j = (t / ntx) * DY + threadIdx.y;
        if (i >= Nx || j >= Ny) continue;
        const double p = phi[cidx(i, j, Nx)];
        const double dx = (i + 0.5) * (P.g.Lx / Nx) - xc, dy = (j + 0.5) * (P.g.Ly / Ny) - yc;
        const double mw = area * p;
        S[0] += mw * dx * dx;
        S[1] += mw * dy * dy;
        S[2] += mw * dx * dy;
        if (cfg.nmax > 0) {
            const double gx = 0.5 * phi_grad_x(P, phi, i, j) + 0.5 * phi_grad_x(P, phi, i + 1, j);
            const double gy = 0.5 * phi_grad_y(P, phi, i, j) + 0.5 * phi_grad_y(P, phi, i, j + 1);
            const double iw = area * hypot(gx, gy);
            const double th = atan2(dy, dx);
            for (int n = 1; n <= cfg.nmax; ++n) {
                double sn, cs;
                sincos(n * th, &sn, &cs);
                S[3 + n - 1] += iw * cs / kPi;
                S[3 + EFSI_DIAG_MAX_MODES + n - 1] += iw * sn / kPi;
            }
        }
    }
    double ts[kDiagSums2];
    if (grid_reduce<kDiagSums2>(S, rs, ts, sh) && threadIdx.x == 0 && threadIdx.y == 0)
        for (int k = 0; k < kDiagSums2; ++k) tot[kDiagSums + kDiagMaxes + k] = ts[k];
}
}  // namespace

void launch_diagnostics(const Params& P, const efsi_diag_config& cfg, const double* U, const double* V,
                        const double* phi, const double* sxx, const double* syy, const double* sxy,
                        const RedSlot& r1, const RedSlot& r2, const RedSlot& r3, double* tot, int max_blocks,
                        cudaStream_t s) {
    const int nt = ((P.g.Nx + DX - 1) / DX) * ((P.g.Ny + DY - 1) / DY);
    const int grid = std::min(persistent_grid(nt, P.nsm, 4), max_blocks);
    k_diag1<<<grid, dim3(DX, DY), 0, s>>>(P, cfg, U, V, phi, sxx, syy, sxy, r1, r2, tot);
    k_diag2<<<grid, dim3(DX, DY), 0, s>>>(P, cfg, phi, r3, tot);
}

}  // namespace efsi
