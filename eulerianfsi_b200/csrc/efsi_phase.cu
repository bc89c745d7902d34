// efsi_phase.cu — conservative phase-field right-hand sides on sm_100a:
// CDI (InterfaceRegularization.jl:123-228 + InterfaceTransport.jl:237-276),
// ACDI (PhaseFieldMethods.jl:479-671) and UWCDI (PhaseFieldMethods.jl:233-404,
// :675-767, :852-867), plus plain upwind transport.
//
// One 32x8 thread block owns a 32x8 tile of cells.  The phase field (and psi for
// ACDI, the smoothed field for UWCDI smoothed9) is staged in shared memory with a
// 3-cell halo, cell-centred normals are computed once per cell for the tile plus
// a 1-cell ring, and each thread then assembles the face fluxes of its cell.  The
// transcendentals (ACDI log per cell, tanh per face) are therefore evaluated once
// per cell instead of once per stencil reference.
#include <cmath>

#include "efsi_kernels.cuh"

namespace efsi {

namespace {
constexpr int TX = 32, TY = 8, H = 3;
constexpr int SX = TX + 2 * H, SY = TY + 2 * H;  // staged field tile
constexpr int NX = TX + 2, NY = TY + 2;          // normals tile (1-cell ring)
}  // namespace

// _phase_boundary_value (PhaseFieldMethods.jl:174-196): homogeneous Neumann /
// outflow faces return the interior value (nonhomogeneous Neumann is rejected when
// the context is created).
__device__ __forceinline__ double pbv(const SideD& s, int k, double interior) {
    if (bdir(s, k)) return bval(s, k);
    return interior;
}

// AXIS = 0: the phase-field right-hand side.  AXIS = 1 / 2: one directional sweep of
// uwcdi_strang_step (PhaseFieldMethods.jl:810-850): out = phi - h div_x(F) (or div_y),
// the flux of the other direction set to zero and no source term.
template <int METHOD, int AXIS = 0>
__global__ void __launch_bounds__(TX* TY) k_phase(Params P, const double* __restrict__ U, const double* __restrict__ V,
                                                  const double* __restrict__ phi, const double* __restrict__ G,
                                                  const double* __restrict__ gamma_dyn, double* out,
                                                  DevStatus* st, double h = 0.0) {
    __shared__ double s_phi[SY][SX];
    __shared__ double s_aux[SY][SX];
    __shared__ double s_nx[NY][NX];
    __shared__ double s_ny[NY][NX];
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool px = P.g.px, py = P.g.py;
    const double ihx = P.g.ihx, ihy = P.g.ihy;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int tid = threadIdx.x + threadIdx.y * TX;
    const double* psi_bc = P.psi_bc;
    const efsi_models& md = P.md;
    const bool smooth9 = METHOD == EFSI_PF_UWCDI && md.pf_option == EFSI_NORMALS_SMOOTHED9;

    // -- stage phi (and psi) -------------------------------------------------------------
    for (int t = tid; t < SX * SY; t += TX * TY) {
        int a = t % SX, b = t / SX;
        int gi = i0 - H + a, gj = j0 - H + b;
        bool valid = true;
        if (px) gi = wrapm(gi, Nx); else valid &= (gi >= 0 && gi < Nx);
        if (py) gj = wrapm(gj, Ny); else valid &= (gj >= 0 && gj < Ny);
        double p = valid ? phi[cidx(gi, gj, Nx)] : 0.0;
        s_phi[b][a] = p;
        if (METHOD == EFSI_PF_ACDI) {
            // psi = eps*log((p+e)/(1-p+e)), p clamped to [0,1] (:479-483)
            double q = clamp01(p), e = md.pf_param[2];
            s_aux[b][a] = valid ? md.pf_param[1] * log((q + e) / (1.0 - q + e)) : 0.0;
        }
    }
    __syncthreads();
    if (smooth9) {  // _smoothed9_field (:377-397), clamp-to-edge indices at walls
        for (int t = tid; t < SX * SY; t += TX * TY) {
            int a = t % SX, b = t / SX;
            if (a == 0 || b == 0 || a == SX - 1 || b == SY - 1) continue;
            int gi = i0 - H + a, gj = j0 - H + b;
            if ((!px && (gi < 0 || gi >= Nx)) || (!py && (gj < 0 || gj >= Ny))) { s_aux[b][a] = 0.0; continue; }
            auto at = [&](int da, int db) {
                int ga = gi + da, gb = gj + db, aa = a + da, bb = b + db;
                if (!px) { if (ga < 0) aa += 1; if (ga >= Nx) aa -= 1; }
                if (!py) { if (gb < 0) bb += 1; if (gb >= Ny) bb -= 1; }
                return s_phi[bb][aa];
            };
            s_aux[b][a] = 0.25 * at(0, 0) + 0.125 * (at(1, 0) + at(-1, 0) + at(0, 1) + at(0, -1)) +
                          0.0625 * (at(1, 1) + at(-1, 1) + at(1, -1) + at(-1, -1));
        }
        __syncthreads();
    }

    // -- centred normals (or the CDI sharpening vector) on tile + 1 ring -----------------
    if (METHOD != EFSI_PF_UPWIND) {
        for (int t = tid; t < NX * NY; t += TX * TY) {
            int a = t % NX, b = t / NX;           // normals coords
            int sa = a + H - 1, sb = b + H - 1;   // staged coords
            int gi = i0 - 1 + a, gj = j0 - 1 + b;
            if ((!px && (gi < 0 || gi >= Nx)) || (!py && (gj < 0 || gj >= Ny))) {
                s_nx[b][a] = 0.0; s_ny[b][a] = 0.0;
                continue;
            }
            int ci = px ? wrapm(gi, Nx) : gi, cj = py ? wrapm(gj, Ny) : gj;
            const double(*F)[SX] = (METHOD == EFSI_PF_ACDI || smooth9) ? s_aux : s_phi;
            // face gradients of F at the four faces of the cell
            auto fgx = [&](bool right) -> double {
                if (!px && (right ? ci == Nx - 1 : ci == 0)) {
                    double in = F[sb][sa];
                    if (METHOD == EFSI_PF_ACDI) {
                        const int side = right ? RIGHT : LEFT;
                        if (P.bphi.s[side].type == EFSI_BC_DIRICHLET)
                            return right ? (psi_bc[side] - in) / (0.5 * P.g.hx) : (in - psi_bc[side]) / (0.5 * P.g.hx);
                        return 0.0;
                    }
                    const SideD& s = P.bphi.s[right ? RIGHT : LEFT];
                    double dist = 0.5 * P.g.hx;
                    if (bdir(s, cj)) return right ? bval(s, cj) / dist - in / dist : in / dist - bval(s, cj) / dist;
                    if (s.type == EFSI_BC_NEUMANN) return (right ? 1.0 : -1.0) * bval(s, cj);
                    if (s.type == EFSI_BC_MIXED) return (right ? 1.0 : -1.0) * bneu(s, cj);
                    return 0.0;
                }
                return right ? (F[sb][sa + 1] - F[sb][sa]) * ihx : (F[sb][sa] - F[sb][sa - 1]) * ihx;
            };
            auto fgy = [&](bool top) -> double {
                if (!py && (top ? cj == Ny - 1 : cj == 0)) {
                    double in = F[sb][sa];
                    if (METHOD == EFSI_PF_ACDI) {
                        const int side = top ? TOP : BOTTOM;
                        if (P.bphi.s[side].type == EFSI_BC_DIRICHLET)
                            return top ? (psi_bc[side] - in) / (0.5 * P.g.hy) : (in - psi_bc[side]) / (0.5 * P.g.hy);
                        return 0.0;
                    }
                    const SideD& s = P.bphi.s[top ? TOP : BOTTOM];
                    double dist = 0.5 * P.g.hy;
                    if (bdir(s, ci)) return top ? bval(s, ci) / dist - in / dist : in / dist - bval(s, ci) / dist;
                    if (s.type == EFSI_BC_NEUMANN) return (top ? 1.0 : -1.0) * bval(s, ci);
                    if (s.type == EFSI_BC_MIXED) return (top ? 1.0 : -1.0) * bneu(s, ci);
                    return 0.0;
                }
                return top ? (F[sb + 1][sa] - F[sb][sa]) * ihy : (F[sb][sa] - F[sb - 1][sa]) * ihy;
            };
            double gx = 0.5 * fgx(false) + 0.5 * fgx(true);
            double gy = 0.5 * fgy(false) + 0.5 * fgy(true);
            if (METHOD == EFSI_PF_UWCDI && md.pf_option == EFSI_NORMALS_YOUNGS &&
                !((!px && (ci == 0 || ci == Nx - 1)) || (!py && (cj == 0 || cj == Ny - 1)))) {
                // Youngs 3x3 gradient (:307-334)
                auto f = [&](int da, int db) { return s_phi[sb + db][sa + da]; };
                gx = (f(1, -1) + 2.0 * f(1, 0) + f(1, 1) - f(-1, -1) - 2.0 * f(-1, 0) - f(-1, 1)) / (8.0 * P.g.hx);
                gy = (f(-1, 1) + 2.0 * f(0, 1) + f(1, 1) - f(-1, -1) - 2.0 * f(0, -1) - f(1, -1)) / (8.0 * P.g.hy);
            }
            double delta = METHOD == EFSI_PF_CDI ? md.pf_param[2] : (METHOD == EFSI_PF_ACDI ? md.pf_param[3] : md.pf_param[1]);
            double mag = sqrt(gx * gx + gy * gy + delta * delta);
            if (METHOD == EFSI_PF_CDI) {  // sharpening vector phi(1-phi) n (InterfaceRegularization.jl:123-145)
                double p = s_phi[sb][sa];
                double amp = p * (1.0 - p);
                s_nx[b][a] = amp * gx / mag;
                s_ny[b][a] = amp * gy / mag;
            } else {
                s_nx[b][a] = gx / mag;
                s_ny[b][a] = gy / mag;
            }
        }
        __syncthreads();
    }

    // -- face fluxes and the cell right-hand side ---------------------------------------------
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    if (i >= Nx || j >= Ny) return;
    const int sa = threadIdx.x + H, sb = threadIdx.y + H;  // staged coords of the cell
    const int na = threadIdx.x + 1, nb = threadIdx.y + 1;  // normals coords of the cell
    const double pc = s_phi[sb][sa];
    const double S = G ? G[cidx(i, j, Nx)] : 0.0;

    // Face f of the cell: dir 0 = x (left f=i, right f=i+1), dir 1 = y.
    // (lo, hi) = staged neighbours across the face; boundary = non-periodic wall face.
    double conv[2][2], reg[2][2];
    for (int dir = 0; dir < 2; ++dir) {
        for (int side = 0; side < 2; ++side) {
            const int f = dir == 0 ? i + side : j + side;
            const int n = dir == 0 ? Nx : Ny;
            const bool per = dir == 0 ? px : py;
            const bool wall = !per && (f == 0 || f == n);
            // staged coordinates of the low / high cell across face f
            int la = sa, lb = sb, ha = sa, hb = sb;
            if (dir == 0) { la = sa + side - 1; ha = sa + side; } else { lb = sb + side - 1; hb = sb + side; }
            const double plo = s_phi[lb][la], phi_hi = s_phi[hb][ha];
            // normal velocity on the face (periodic duplicate face n reads face 0)
            double vel;
            if (dir == 0) vel = U[uidx((per && f == n) ? 0 : f, j, Nx)];
            else vel = V[vidx(i, (per && f == n) ? 0 : f, Nx)];
            const SideD* wside = nullptr;
            if (wall) wside = dir == 0 ? &P.bphi.s[f == 0 ? LEFT : RIGHT] : &P.bphi.s[f == 0 ? BOTTOM : TOP];
            const int wk = dir == 0 ? j : i;  // boundary data index along the wall
            const double h_i = dir == 0 ? ihx : ihy;
            double cflux = 0.0, rflux = 0.0;
            if (METHOD == EFSI_PF_ACDI) {
                double pf = wall ? pbv(*wside, wk, f == 0 ? phi_hi : plo) : 0.5 * plo + 0.5 * phi_hi;
                cflux = vel * pf;
                if (!wall) {
                    double geff = md.pf_option ? *gamma_dyn : md.pf_param[0];
                    double eps = md.pf_param[1];
                    double psf = 0.5 * s_aux[lb][la] + 0.5 * s_aux[hb][ha];
                    double th = tanh(psf / (2.0 * eps));
                    double amp = 0.25 * (1.0 - th * th);
                    int nla = la - H + 1, nlb = lb - H + 1, nha = ha - H + 1, nhb = hb - H + 1;
                    double nf = dir == 0 ? 0.5 * s_nx[nlb][nla] + 0.5 * s_nx[nhb][nha]
                                         : 0.5 * s_ny[nlb][nla] + 0.5 * s_ny[nhb][nha];
                    rflux = geff * (eps * ((phi_hi - plo) * h_i) - amp * nf);
                }
            } else if (METHOD == EFSI_PF_UWCDI) {
                double up;
                int nla, nlb, nha, nhb;
                if (wall) {
                    bool lowwall = f == 0;
                    double in = lowwall ? phi_hi : plo;
                    double b = pbv(*wside, wk, in);
                    up = lowwall ? (vel >= 0.0 ? b : in) : (vel >= 0.0 ? in : b);
                    int ca = lowwall ? ha : la, cb = lowwall ? hb : lb;
                    nla = nha = ca - H + 1; nlb = nhb = cb - H + 1;
                } else {
                    up = vel >= 0.0 ? plo : phi_hi;
                    nla = la - H + 1; nlb = lb - H + 1; nha = ha - H + 1; nhb = hb - H + 1;
                }
                double nn, nt;  // normal / transverse interpolated components
                if (nla == nha && nlb == nhb) {
                    nn = dir == 0 ? s_nx[nlb][nla] : s_ny[nlb][nla];
                    nt = dir == 0 ? s_ny[nlb][nla] : s_nx[nlb][nla];
                } else if (dir == 0) {
                    nn = 0.5 * s_nx[nlb][nla] + 0.5 * s_nx[nhb][nha];
                    nt = 0.5 * s_ny[nlb][nla] + 0.5 * s_ny[nhb][nha];
                } else {
                    nn = 0.5 * s_ny[nlb][nla] + 0.5 * s_ny[nhb][nha];
                    nt = 0.5 * s_nx[nlb][nla] + 0.5 * s_nx[nhb][nha];
                }
                double delta = md.pf_param[1];
                double nf = nn / sqrt(nn * nn + nt * nt + delta * delta);
                double ratio = dir == 0 ? P.g.hy / P.g.hx : P.g.hx / P.g.hy;
                double alpha = md.pf_param[0] * fmax(1.0, ratio);
                double beta = fabs(vel) / alpha;
                cflux = up * (vel + beta * nf * (1.0 - up));
            } else {  // CDI and plain upwind: first-order upwind material flux
                double up;
                if (wall) {
                    bool lowwall = f == 0;
                    double in = lowwall ? phi_hi : plo;
                    double b = in;
                    if (vel != 0.0 && (lowwall ? vel > 0.0 : vel < 0.0)) {  // inflow
                        if (wside->type == EFSI_BC_DIRICHLET) b = bval(*wside, wk);
                        else raise_err(st, DE_NEUMANN_INFLOW, 2, i, j, vel);
                    }
                    up = lowwall ? (vel >= 0.0 ? b : in) : (vel >= 0.0 ? in : b);
                } else {
                    up = vel >= 0.0 ? plo : phi_hi;
                }
                cflux = vel * up;
                if (METHOD == EFSI_PF_CDI && !wall) {
                    int nla = la - H + 1, nlb = lb - H + 1, nha = ha - H + 1, nhb = hb - H + 1;
                    double sf = dir == 0 ? 0.5 * s_nx[nlb][nla] + 0.5 * s_nx[nhb][nha]
                                         : 0.5 * s_ny[nlb][nla] + 0.5 * s_ny[nhb][nha];
                    double ell = 0.5 * md.pf_param[1];
                    rflux = md.pf_param[0] * (sf - ell * ((phi_hi - plo) * h_i));
                }
            }
            conv[dir][side] = cflux;
            reg[dir][side] = rflux;
        }
    }
    if (AXIS != 0) {
        const double d = AXIS == 1 ? (conv[0][1] - conv[0][0]) * ihx : (conv[1][1] - conv[1][0]) * ihy;
        out[cidx(i, j, Nx)] = pc + h * (-d);
        return;
    }
    double divc = (conv[0][1] - conv[0][0]) * ihx + (conv[1][1] - conv[1][0]) * ihy;
    double divr = (reg[0][1] - reg[0][0]) * ihx + (reg[1][1] - reg[1][0]) * ihy;
    double r;
    if (METHOD == EFSI_PF_ACDI) r = -divc + divr + pc * S;           // :668-670
    else if (METHOD == EFSI_PF_CDI) r = -divc - divr + pc * S;       // InterfaceTransport.jl:274-275
    else r = -divc + pc * S;                                          // :866 and the upwind path
    out[cidx(i, j, Nx)] = r;
}

void launch_phase_rhs(const Params& P, const StageFields& f, const double* gamma_eff, double* Ephi, DevStatus* st,
                      cudaStream_t s) {
    dim3 grid((P.g.Nx + TX - 1) / TX, (P.g.Ny + TY - 1) / TY), block(TX, TY);
    switch (P.md.phase_field_method) {
        case EFSI_PF_ACDI:
            k_phase<EFSI_PF_ACDI><<<grid, block, 0, s>>>(P, f.U, f.V, f.phi, f.G, gamma_eff, Ephi, st);
            break;
        case EFSI_PF_UWCDI:
            k_phase<EFSI_PF_UWCDI><<<grid, block, 0, s>>>(P, f.U, f.V, f.phi, f.G, gamma_eff, Ephi, st);
            break;
        case EFSI_PF_CDI:
            k_phase<EFSI_PF_CDI><<<grid, block, 0, s>>>(P, f.U, f.V, f.phi, f.G, gamma_eff, Ephi, st);
            break;
        default:
            k_phase<EFSI_PF_UPWIND><<<grid, block, 0, s>>>(P, f.U, f.V, f.phi, f.G, gamma_eff, Ephi, st);
            break;
    }
}

void launch_strang_sweep(const Params& P, const double* U, const double* V, const double* phi, double* out, int axis,
                         double h, DevStatus* st, cudaStream_t s) {
    dim3 grid((P.g.Nx + TX - 1) / TX, (P.g.Ny + TY - 1) / TY), block(TX, TY);
    if (axis == 1)
        k_phase<EFSI_PF_UWCDI, 1><<<grid, block, 0, s>>>(P, U, V, phi, nullptr, nullptr, out, st, h);
    else
        k_phase<EFSI_PF_UWCDI, 2><<<grid, block, 0, s>>>(P, U, V, phi, nullptr, nullptr, out, st, h);
}

}  // namespace efsi
