// efsi_adjoint.cu — discrete adjoint of the IMEX step on sm_100a: the transposed
// Jacobians of the explicit tendencies, the transposed projection right-hand side and
// correction, and the transposed stage combinations.  The adjoint solves reuse the SPD
// forward solvers (efsi_solvers.cu); the orchestration of a reverse step lives in
// efsi_api.cu.
//
// Transposed stencils are formed from local Jacobian rows: each thread owns one output
// point of a forward operator (a MAC face or a cell), re-evaluates the forward point
// function with forward-mode numbers seeded on the inputs it reads, and scatters
// lambda_out * d(out)/d(input) into the input adjoints with atomics.  The point
// functions below restate the forward helpers of efsi_ops.cu / efsi_phase.cu branch for
// branch (walls, periodic wrap, boundary data), so the transpose is exact for every
// boundary variant.  Where an operator is a chain of local maps (the ACDI flux: psi ->
// cell normal -> face flux), each link is reversed separately through scratch arrays,
// which keeps every forward-mode number short.  Atomic accumulation makes the adjoint
// reproducible to round-off, not bit for bit.
#include <cmath>

#include "efsi_adjoint.cuh"
#include "efsi_device.cuh"

namespace efsi {
namespace {

constexpr int BX = 32, BY = 8;
inline dim3 grid2(int nx, int ny) { return dim3((nx + BX - 1) / BX, (ny + BY - 1) / BY); }

__constant__ double a_AE[4][4] = {{0, 0, 0, 0}, {8.0 / 15, 0, 0, 0}, {1.0 / 4, 5.0 / 12, 0, 0}, {1.0 / 4, 0, 3.0 / 4, 0}};
__constant__ double a_AI[4][4] = {{0, 0, 0, 0}, {4.0 / 15, 4.0 / 15, 0, 0}, {4.0 / 15, 1.0 / 3, 1.0 / 15, 0},
                                  {4.0 / 15, 1.0 / 3, 7.0 / 30, 1.0 / 6}};

// ---- forward-mode numbers: value and K partial derivatives ---------------------------------
template <int K>
struct Dn {
    double v;
    double d[K];
};
template <int K>
__device__ __forceinline__ Dn<K> dconst(double v) {
    Dn<K> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = 0.0;
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> dseed(double v, int s) {
    Dn<K> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (k == s) ? 1.0 : 0.0;
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator+(const Dn<K>& a, const Dn<K>& b) {
    Dn<K> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator-(const Dn<K>& a, const Dn<K>& b) {
    Dn<K> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator-(const Dn<K>& a) {
    Dn<K> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator*(const Dn<K>& a, const Dn<K>& b) {
    Dn<K> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator/(const Dn<K>& a, const Dn<K>& b) {
    Dn<K> r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator+(const Dn<K>& a, double b) {
    Dn<K> r = a;
    r.v = a.v + b;
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator+(double a, const Dn<K>& b) {
    Dn<K> r = b;
    r.v = a + b.v;
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator-(const Dn<K>& a, double b) {
    Dn<K> r = a;
    r.v = a.v - b;
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator-(double a, const Dn<K>& b) {
    Dn<K> r;
    r.v = a - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator*(const Dn<K>& a, double b) {
    Dn<K> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> operator*(double a, const Dn<K>& b) {
    return b * a;
}
template <int K>
__device__ __forceinline__ Dn<K> operator/(const Dn<K>& a, double b) {
    Dn<K> r;
    r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] / b;
    return r;
}
// Elementary functions: CUDA's function for the value, the derivative from calculus.
template <int K>
__device__ __forceinline__ Dn<K> dsqrt(const Dn<K>& a) {
    Dn<K> r;
    r.v = sqrt(a.v);
    const double g = r.v > 0.0 ? 0.5 / r.v : 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = g * a.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> dlog(const Dn<K>& a) {
    Dn<K> r;
    r.v = log(a.v);
    const double g = 1.0 / a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = g * a.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> dpow(const Dn<K>& a, double p) {
    Dn<K> r;
    r.v = pow(a.v, p);
    const double g = a.v != 0.0 ? p * pow(a.v, p - 1.0) : (p == 1.0 ? 1.0 : 0.0);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = g * a.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> dhypot(const Dn<K>& a, const Dn<K>& b) {
    Dn<K> r;
    r.v = hypot(a.v, b.v);
    const double ia = r.v > 0.0 ? a.v / r.v : 0.0, ib = r.v > 0.0 ? b.v / r.v : 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = ia * a.d[k] + ib * b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dn<K> dlog1p(const Dn<K>& a) {
    Dn<K> r;
    r.v = log1p(a.v);
    const double g = 1.0 / (1.0 + a.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = g * a.d[k];
    return r;
}
// sech^2(x) = 1 - tanh^2(x) from e = exp(-2|x|): 4e / (1 + e)^2 keeps its full relative
// accuracy where it is tiny (|x| large), unlike the difference 1 - tanh^2, whose rounding
// error there is larger than the value itself.
template <int K>
__device__ __forceinline__ Dn<K> dsech2(const Dn<K>& a) {
    Dn<K> r;
    const double e = exp(-2.0 * fabs(a.v));
    const double den = 1.0 + e;
    r.v = 4.0 * e / (den * den);
    const double th = (a.v >= 0.0 ? 1.0 : -1.0) * (1.0 - e) / den;  // tanh(x)
    const double g = -2.0 * th * r.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = g * a.d[k];
    return r;
}
// clamp to [0, 1]: slope 1 inside, 0 outside
template <int K>
__device__ __forceinline__ Dn<K> dclamp01(const Dn<K>& a) {
    if (a.v < 0.0) return dconst<K>(0.0);
    if (a.v > 1.0) return dconst<K>(1.0);
    return a;
}

// ---- the inputs a point function reads ----------------------------------------------------
// Every adjoint array an operator scatters into has a tag; a point function records each
// distinct (tag, index) it reads as one seed of its forward-mode numbers.
enum Tag : int {
    T_U = 0, T_V, T_PHI, T_SXX, T_SYY, T_SXY,
    T_BUB, T_BUT, T_BVL, T_BVR,     // tangential wall velocity data
    T_TXX, T_TYY, T_TXY,            // cell stresses of the stress divergence
    T_COUNT
};
struct Lam {
    double* p[T_COUNT];
};

template <int K>
struct Rec {
    int n;
    int over;
    int tag[K];
    int idx[K];
    __device__ __forceinline__ void init() { n = 0; over = 0; }
    __device__ Dn<K> in(int t, int i, double v) {
        for (int s = 0; s < n; ++s)
            if (tag[s] == t && idx[s] == i) return dseed<K>(v, s);
        if (n >= K) { over = 1; return dconst<K>(v); }
        tag[n] = t;
        idx[n] = i;
        return dseed<K>(v, n++);
    }
};

// lam_in[input] += lam * d(out)/d(input) for every recorded input.
template <int K>
__device__ __forceinline__ void scatter(const Rec<K>& r, const Dn<K>& out, double lam, const Lam& L) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (k < r.n) {
            const double g = out.d[k] * lam;
            double* a = L.p[r.tag[k]];
            if (g != 0.0 && a) atomicAdd(a + r.idx[k], g);
        }
    }
}

__device__ __forceinline__ void overflow(DevStatus* st, int where, int i, int j) {
    // a point function read more inputs than its forward-mode numbers hold
    raise_err(st, DE_NONFINITE_INPUT, 100 + where, i, j, 0.0);
}

// =====================================================================================
// Momentum forcing (TimeIntegrationIMEX.jl:959-985): convection and stress divergence
// =====================================================================================
// u_corner / v_corner / conv_x / conv_y of efsi_ops.cu with recorded inputs.
template <int K>
__device__ Dn<K> u_corner_d(const Params& P, const double* U, Rec<K>& r, int i, int jc) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    auto u = [&](int a, int b) {
        const int k = (int)uidx(a, b, Nx);
        return r.in(T_U, k, U[k]);
    };
    const int ii = (P.g.px && i == Nx) ? 0 : i;
    if (P.g.py) {
        if (jc == 0 || jc == Ny) return 0.5 * (u(ii, Ny - 1) + u(ii, 0));
        return 0.5 * (u(ii, jc - 1) + u(ii, jc));
    }
    if (jc == 0 || jc == Ny) {
        const SideD& s = P.bu.s[jc == 0 ? BOTTOM : TOP];
        if (s.type == EFSI_BC_DIRICHLET) return r.in(jc == 0 ? T_BUB : T_BUT, ii, bval(s, ii));
        Dn<K> adj = u(ii, jc == 0 ? 0 : Ny - 1);
        return adj + bval(s, ii) * (0.5 * P.g.hy);
    }
    return 0.5 * (u(ii, jc - 1) + u(ii, jc));
}
template <int K>
__device__ Dn<K> v_corner_d(const Params& P, const double* V, Rec<K>& r, int ic, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    auto v = [&](int a, int b) {
        const int k = (int)vidx(a, b, Nx);
        return r.in(T_V, k, V[k]);
    };
    const int jj = (P.g.py && j == Ny) ? 0 : j;
    if (P.g.px) {
        if (ic == 0 || ic == Nx) return 0.5 * (v(Nx - 1, jj) + v(0, jj));
        return 0.5 * (v(ic - 1, jj) + v(ic, jj));
    }
    if (ic == 0 || ic == Nx) {
        const SideD& s = P.bv.s[ic == 0 ? LEFT : RIGHT];
        if (s.type == EFSI_BC_DIRICHLET) return r.in(ic == 0 ? T_BVL : T_BVR, jj, bval(s, jj));
        Dn<K> adj = v(ic == 0 ? 0 : Nx - 1, jj);
        return adj + bval(s, jj) * (0.5 * P.g.hx);
    }
    return 0.5 * (v(ic - 1, jj) + v(ic, jj));
}
template <int K>
__device__ Dn<K> conv_x_d(const Params& P, const double* U, const double* V, Rec<K>& r, int i, int j) {
    const int Nx = P.g.Nx;
    if (!P.g.px && (i == 0 || i == Nx)) return dconst<K>(0.0);
    const int ic = (i == Nx) ? 0 : i;
    const int im = wrapi(ic - 1, Nx);
    auto u = [&](int a, int b) {
        const int k = (int)uidx(a, b, Nx);
        return r.in(T_U, k, U[k]);
    };
    auto u2 = [&](int c) {
        Dn<K> ur = (P.g.px && c == Nx - 1) ? u(0, j) : u(c + 1, j);
        Dn<K> uc = 0.5 * u(c, j) + 0.5 * ur;
        return uc * uc;
    };
    return (u2(ic) - u2(im)) * P.g.ihx +
           (u_corner_d(P, U, r, ic, j + 1) * v_corner_d(P, V, r, ic, j + 1) -
            u_corner_d(P, U, r, ic, j) * v_corner_d(P, V, r, ic, j)) *
               P.g.ihy;
}
template <int K>
__device__ Dn<K> conv_y_d(const Params& P, const double* U, const double* V, Rec<K>& r, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (!P.g.py && (j == 0 || j == Ny)) return dconst<K>(0.0);
    const int jc = (j == Ny) ? 0 : j;
    const int jm = wrapi(jc - 1, Ny);
    auto v = [&](int a, int b) {
        const int k = (int)vidx(a, b, Nx);
        return r.in(T_V, k, V[k]);
    };
    auto v2 = [&](int c) {
        Dn<K> vt = (P.g.py && c == Ny - 1) ? v(i, 0) : v(i, c + 1);
        Dn<K> vc = 0.5 * v(i, c) + 0.5 * vt;
        return vc * vc;
    };
    return (u_corner_d(P, U, r, i + 1, jc) * v_corner_d(P, V, r, i + 1, jc) -
            u_corner_d(P, U, r, i, jc) * v_corner_d(P, V, r, i, jc)) *
               P.g.ihx +
           (v2(jc) - v2(jm)) * P.g.ihy;
}

// symmetric_stress_divergence (Operators.jl:620-842) as a linear map of the cell stresses.
template <int K>
struct StressIn {
    Rec<K>* r;
    int Nx;
    __device__ __forceinline__ Dn<K> xx(int i, int j) const { return r->in(T_TXX, (int)cidx(i, j, Nx), 0.0); }
    __device__ __forceinline__ Dn<K> yy(int i, int j) const { return r->in(T_TYY, (int)cidx(i, j, Nx), 0.0); }
    __device__ __forceinline__ Dn<K> xy(int i, int j) const { return r->in(T_TXY, (int)cidx(i, j, Nx), 0.0); }
};
template <int K>
__device__ Dn<K> txy_xface_d(const Params& P, const StressIn<K>& c, int i, int r) {
    const int Nx = P.g.Nx;
    if (P.g.px) {
        if (i == 0 || i == Nx) return 0.5 * (c.xy(Nx - 1, r) + c.xy(0, r));
    } else {
        if (i == 0) { Dn<K> a = c.xy(0, r), b = c.xy(1, r); return a - (b - a) * 0.5; }
        if (i == Nx) { Dn<K> a = c.xy(Nx - 1, r), b = c.xy(Nx - 2, r); return a + (a - b) * 0.5; }
    }
    return 0.5 * (c.xy(i - 1, r) + c.xy(i, r));
}
template <int K>
__device__ Dn<K> txy_yface_d(const Params& P, const StressIn<K>& c, int ci, int j) {
    const int Ny = P.g.Ny;
    if (P.g.py) {
        if (j == 0 || j == Ny) return 0.5 * (c.xy(ci, Ny - 1) + c.xy(ci, 0));
    } else {
        if (j == 0) { Dn<K> a = c.xy(ci, 0), b = c.xy(ci, 1); return a - (b - a) * 0.5; }
        if (j == Ny) { Dn<K> a = c.xy(ci, Ny - 1), b = c.xy(ci, Ny - 2); return a + (a - b) * 0.5; }
    }
    return 0.5 * (c.xy(ci, j - 1) + c.xy(ci, j));
}
template <int K>
__device__ Dn<K> ssd_x_d(const Params& P, const StressIn<K>& c, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    Dn<K> dxx;
    if (P.g.px) {
        const int ic = (i == Nx) ? 0 : i;
        dxx = (c.xx(ic, j) - c.xx(wrapi(ic - 1, Nx), j)) * P.g.ihx;
    } else if (i == 0) {
        dxx = (c.xx(1, j) - c.xx(0, j)) * P.g.ihx;
    } else if (i == Nx) {
        dxx = (c.xx(Nx - 1, j) - c.xx(Nx - 2, j)) * P.g.ihx;
    } else {
        dxx = (c.xx(i, j) - c.xx(i - 1, j)) * P.g.ihx;
    }
    Dn<K> dxy;
    if (P.g.py) {
        dxy = (txy_xface_d(P, c, i, wrapi(j + 1, Ny)) - txy_xface_d(P, c, i, wrapi(j - 1, Ny))) / (2.0 * P.g.hy);
    } else if (j == 0) {
        dxy = (txy_xface_d(P, c, i, 1) - txy_xface_d(P, c, i, 0)) * P.g.ihy;
    } else if (j == Ny - 1) {
        dxy = (txy_xface_d(P, c, i, Ny - 1) - txy_xface_d(P, c, i, Ny - 2)) * P.g.ihy;
    } else {
        dxy = (txy_xface_d(P, c, i, j + 1) - txy_xface_d(P, c, i, j - 1)) / (2.0 * P.g.hy);
    }
    return dxx + dxy;
}
template <int K>
__device__ Dn<K> ssd_y_d(const Params& P, const StressIn<K>& c, int i, int j) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    Dn<K> dyy;
    if (P.g.py) {
        const int jc = (j == Ny) ? 0 : j;
        dyy = (c.yy(i, jc) - c.yy(i, wrapi(jc - 1, Ny))) * P.g.ihy;
    } else if (j == 0) {
        dyy = (c.yy(i, 1) - c.yy(i, 0)) * P.g.ihy;
    } else if (j == Ny) {
        dyy = (c.yy(i, Ny - 1) - c.yy(i, Ny - 2)) * P.g.ihy;
    } else {
        dyy = (c.yy(i, j) - c.yy(i, j - 1)) * P.g.ihy;
    }
    Dn<K> dxy;
    if (P.g.px) {
        dxy = (txy_yface_d(P, c, wrapi(i + 1, Nx), j) - txy_yface_d(P, c, wrapi(i - 1, Nx), j)) / (2.0 * P.g.hx);
    } else if (i == 0) {
        dxy = (txy_yface_d(P, c, 1, j) - txy_yface_d(P, c, 0, j)) * P.g.ihx;
    } else if (i == Nx - 1) {
        dxy = (txy_yface_d(P, c, Nx - 1, j) - txy_yface_d(P, c, Nx - 2, j)) * P.g.ihx;
    } else {
        dxy = (txy_yface_d(P, c, i + 1, j) - txy_yface_d(P, c, i - 1, j)) / (2.0 * P.g.hx);
    }
    return dyy + dxy;
}

// E_uv rows (i, j) of the compact vector: lam of -convection into U, V and wall data;
// lam of the stress divergence into the cell-stress scratch.
__global__ void k_adj_momentum(Params P, AdjIn f, const double* __restrict__ lEu, const double* __restrict__ lEv,
                               Lam L, int elastic, DevStatus* st) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    const size_t k = cidx(i, j, Nx);
    const double lu = lEu[k], lv = lEv[k];
    if (lu != 0.0) {
        Rec<14> r;
        r.init();
        Dn<14> c = conv_x_d(P, f.U, f.V, r, i, j);
        scatter(r, c, -lu, L);
        if (r.over) overflow(st, 0, i, j);
        if (elastic) {
            Rec<10> q;
            q.init();
            Dn<10> s = ssd_x_d(P, StressIn<10>{&q, Nx}, i, j);
            scatter(q, s, lu, L);
            if (q.over) overflow(st, 1, i, j);
        }
    }
    if (lv != 0.0) {
        Rec<14> r;
        r.init();
        Dn<14> c = conv_y_d(P, f.U, f.V, r, i, j);
        scatter(r, c, -lv, L);
        if (r.over) overflow(st, 2, i, j);
        if (elastic) {
            Rec<10> q;
            q.init();
            Dn<10> s = ssd_y_d(P, StressIn<10>{&q, Nx}, i, j);
            scatter(q, s, lv, L);
            if (q.over) overflow(st, 3, i, j);
        }
    }
}

// Cell stress phi * G (sigma - I) (_accumulate_elastic_force!, TimeIntegrationIMEX.jl:903-924):
// lam of phi, sigma and G from the cell-stress adjoints.
__global__ void k_adj_tau(Params P, AdjIn f, const double* __restrict__ ltxx, const double* __restrict__ ltyy,
                          const double* __restrict__ ltxy, AdjOut o, double* lamG) {
    __shared__ double sh[32];
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    double acc[1] = {0.0};
    if (i < P.g.Nx && j < P.g.Ny) {
        const size_t k = cidx(i, j, P.g.Nx);
        const double g = P.md.elastic_coefficient, ph = f.phi[k];
        const double ax = ltxx[k], ay = ltyy[k], ac = ltxy[k];
        const double w = ax * (f.sxx[k] - 1.0) + ay * (f.syy[k] - 1.0) + ac * f.sxy[k];
        o.phi[k] += g * w;
        o.sxx[k] += ph * g * ax;
        o.syy[k] += ph * g * ay;
        o.sxy[k] += ph * g * ac;
        acc[0] = ph * w;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0 && lamG && acc[0] != 0.0) atomicAdd(lamG, acc[0]);
}

// =====================================================================================
// Viscous operator I_uv = A uv + b (Operators.jl:929-1083; k_viscous_apply)
// =====================================================================================
// One row of k_viscous_apply's general path for a constant viscosity mu.
template <int K>
__device__ Dn<K> visc_row_d(const Params& P, double mu, const double* U, const double* V, Rec<K>& r, int i, int j,
                            bool urow) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const double ihx = P.g.ihx, ihy = P.g.ihy;
    auto u = [&](int a, int b) {
        const int k = (int)uidx(a, b, Nx);
        return r.in(T_U, k, U[k]);
    };
    auto v = [&](int a, int b) {
        const int k = (int)vidx(a, b, Nx);
        return r.in(T_V, k, V[k]);
    };
    auto txx = [&](int c, int rr) {
        Dn<K> nxt = c < Nx - 1 ? u(c + 1, rr) : (P.g.px ? u(0, rr) : dconst<K>(bval(P.bu.s[RIGHT], rr)));
        return 2.0 * mu * ((nxt - u(c, rr)) * ihx);
    };
    auto tyy = [&](int c, int rr) {
        Dn<K> nxt = rr < Ny - 1 ? v(c, rr + 1) : (P.g.py ? v(c, 0) : dconst<K>(bval(P.bv.s[TOP], c)));
        return 2.0 * mu * ((nxt - v(c, rr)) * ihy);
    };
    auto txy = [&](int c, int rr) {
        Dn<K> duy = rr > 0 ? (u(c, rr) - u(c, rr - 1)) * ihy
                           : (P.g.py ? (u(c, 0) - u(c, Ny - 1)) * ihy : dconst<K>(0.0));
        Dn<K> dvx = c > 0 ? (v(c, rr) - v(c - 1, rr)) * ihx
                          : (P.g.px ? (v(0, rr) - v(Nx - 1, rr)) * ihx : dconst<K>(0.0));
        return 2.0 * mu * (0.5 * duy + 0.5 * dvx);
    };
    if (urow) {
        Dn<K> axx = txx(i, j) - (i > 0 ? txx(i - 1, j) : (P.g.px ? txx(Nx - 1, j) : dconst<K>(0.0)));
        Dn<K> axy = -txy(i, j) + (j < Ny - 1 ? txy(i, j + 1) : (P.g.py ? txy(i, 0) : dconst<K>(0.0)));
        Dn<K> au = axx * ihx + axy * ihy;
        if (!P.g.py) {
            if (j == 0 && P.bu.s[BOTTOM].type == EFSI_BC_DIRICHLET) {
                const double w = mu / (P.g.hy * (0.5 * P.g.hy));
                au = au + (-w * u(i, 0) + w * r.in(T_BUB, i, bval(P.bu.s[BOTTOM], i)));
            }
            if (j == Ny - 1 && P.bu.s[TOP].type == EFSI_BC_DIRICHLET) {
                const double w = mu / (P.g.hy * (0.5 * P.g.hy));
                au = au + (-w * u(i, Ny - 1) + w * r.in(T_BUT, i, bval(P.bu.s[TOP], i)));
            }
        }
        return au;
    }
    Dn<K> ayx = -txy(i, j) + (i < Nx - 1 ? txy(i + 1, j) : (P.g.px ? txy(0, j) : dconst<K>(0.0)));
    Dn<K> ayy = tyy(i, j) - (j > 0 ? tyy(i, j - 1) : (P.g.py ? tyy(i, Ny - 1) : dconst<K>(0.0)));
    Dn<K> av = ayx * ihx + ayy * ihy;
    if (!P.g.px) {
        if (i == 0 && P.bv.s[LEFT].type == EFSI_BC_DIRICHLET) {
            const double w = mu / (P.g.hx * (0.5 * P.g.hx));
            av = av + (-w * v(0, j) + w * r.in(T_BVL, j, bval(P.bv.s[LEFT], j)));
        }
        if (i == Nx - 1 && P.bv.s[RIGHT].type == EFSI_BC_DIRICHLET) {
            const double w = mu / (P.g.hx * (0.5 * P.g.hx));
            av = av + (-w * v(Nx - 1, j) + w * r.in(T_BVR, j, bval(P.bv.s[RIGHT], j)));
        }
    }
    return av;
}

__global__ void k_adj_visc(Params P, AdjIn f, const double* __restrict__ lIu, const double* __restrict__ lIv, Lam L,
                           DevStatus* st) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    const size_t k = cidx(i, j, Nx);
    const double mu = P.md.viscosity_fluid;
    const double lu = lIu[k], lv = lIv[k];
    if (lu != 0.0) {
        Rec<14> r;
        r.init();
        Dn<14> a = visc_row_d(P, mu, f.U, f.V, r, i, j, true);
        scatter(r, a, lu, L);
        if (r.over) overflow(st, 4, i, j);
    }
    if (lv != 0.0) {
        Rec<14> r;
        r.init();
        Dn<14> a = visc_row_d(P, mu, f.U, f.V, r, i, j, false);
        scatter(r, a, lv, L);
        if (r.over) overflow(st, 5, i, j);
    }
}

// =====================================================================================
// ACDI phase-field right-hand side (PhaseFieldMethods.jl:479-671; k_phase<ACDI>)
// =====================================================================================
__device__ __forceinline__ double acdi_psi(const efsi_models& md, double p) {
    const double q = clamp01(p), e = md.pf_param[2];
    return md.pf_param[1] * log((q + e) / (1.0 - q + e));
}
#ifndef EFSI_ADJ_NORMAL_FLOOR
#define EFSI_ADJ_NORMAL_FLOOR 1e-6
#endif
#ifndef EFSI_ADJ_PSI_SLOPE_FLOOR
#define EFSI_ADJ_PSI_SLOPE_FLOOR 1e-8
#endif
// d(psi)/d(phi) as the reverse sweep uses it.  psi saturates on the plateaus phi <= 0 and
// phi >= 1 (the clamp), which take the clamp's zero slope.  Inside (0, 1) the slope
// eps (1/(q + e) + 1/(1 - q + e)) reaches eps / min(q, 1 - q) next to the plateaus: cells
// of the disk interior at phi = 1 - 1e-16 give 1e13 eps, where the forward map, whose phi
// resolves 1 - phi to a few bits, responds to no admissible perturbation, while the
// reverse sweep multiplies every adjoint through it (1e30 per step at 256^2 measured).
// The slope is therefore taken with the floor max(e, EFSI_ADJ_PSI_SLOPE_FLOOR).
__device__ __forceinline__ double acdi_dpsi(const efsi_models& md, double p) {
    if (!(p > 0.0 && p < 1.0)) return 0.0;
    const double e = fmax(md.pf_param[2], EFSI_ADJ_PSI_SLOPE_FLOOR);
    return md.pf_param[1] * (1.0 / (p + e) + 1.0 / (1.0 - p + e));
}

// Cell normal from psi at the cell and its four neighbours (the face-gradient rules of
// k_phase at walls: Dirichlet phase sides use the side's psi, others a zero gradient).
// Slots: 0 centre, 1 west, 2 east, 3 south, 4 north.
__device__ void acdi_normal_d(const Params& P, const double* psi, int ci, int cj, Dn<5>& nx, Dn<5>& ny,
                              int (&nb)[5]) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool px = P.g.px, py = P.g.py;
    nb[0] = (int)cidx(ci, cj, Nx);
    nb[1] = (px || ci > 0) ? (int)cidx(wrapi(ci - 1, Nx), cj, Nx) : -1;
    nb[2] = (px || ci < Nx - 1) ? (int)cidx(wrapi(ci + 1, Nx), cj, Nx) : -1;
    nb[3] = (py || cj > 0) ? (int)cidx(ci, wrapi(cj - 1, Ny), Nx) : -1;
    nb[4] = (py || cj < Ny - 1) ? (int)cidx(ci, wrapi(cj + 1, Ny), Nx) : -1;
    Dn<5> c = dseed<5>(psi[nb[0]], 0);
    auto at = [&](int s) { return dseed<5>(psi[nb[s]], s); };
    auto wall = [&](int side, bool high, double h) {  // face gradient at a wall face
        if (P.bphi.s[side].type == EFSI_BC_DIRICHLET)
            return high ? (P.psi_bc[side] - c) / (0.5 * h) : (c - P.psi_bc[side]) / (0.5 * h);
        return dconst<5>(0.0);
    };
    Dn<5> gl = nb[1] >= 0 ? (c - at(1)) * P.g.ihx : wall(LEFT, false, P.g.hx);
    Dn<5> gr = nb[2] >= 0 ? (at(2) - c) * P.g.ihx : wall(RIGHT, true, P.g.hx);
    Dn<5> gb = nb[3] >= 0 ? (c - at(3)) * P.g.ihy : wall(BOTTOM, false, P.g.hy);
    Dn<5> gt = nb[4] >= 0 ? (at(4) - c) * P.g.ihy : wall(TOP, true, P.g.hy);
    Dn<5> gx = 0.5 * gl + 0.5 * gr;
    Dn<5> gy = 0.5 * gb + 0.5 * gt;
    // value: g / sqrt(|g|^2 + delta^2) as the forward has it.  Derivative: the same map
    // with the gradient floor max(delta, EFSI_ADJ_NORMAL_FLOOR); where psi is flat (the
    // saturated disk interior, whose rounded phi makes neighbouring psi equal) the
    // forward's 1/delta = 1e14 sensitivity meets flux amplitudes of 1e-16 and would close
    // a loop in the reverse sweep that grows without bound.
    const double delta = P.md.pf_param[3];
    const double da = fmax(delta, EFSI_ADJ_NORMAL_FLOOR);
    const double g2 = gx.v * gx.v + gy.v * gy.v;
    const double m = sqrt(g2 + delta * delta), ma = sqrt(g2 + da * da);
    nx.v = gx.v / m;
    ny.v = gy.v / m;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const double dm = (gx.v * gx.d[k] + gy.v * gy.d[k]) / ma;
        nx.d[k] = (gx.d[k] - gx.v / ma * dm) / ma;
        ny.d[k] = (gy.d[k] - gy.v / ma * dm) / ma;
    }
}

// psi and the cell normals of the stage field; clears the layer adjoints.
__global__ void k_adj_acdi_cells(Params P, const double* __restrict__ phi, AdjScratch s) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= P.g.Nx || j >= P.g.Ny) return;
    const size_t k = cidx(i, j, P.g.Nx);
    s.psi[k] = acdi_psi(P.md, phi[k]);
    s.lpsi[k] = 0.0;
    s.lnx[k] = 0.0;
    s.lny[k] = 0.0;
}
__global__ void k_adj_acdi_normals(Params P, AdjScratch s) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= P.g.Nx || j >= P.g.Ny) return;
    Dn<5> nx, ny;
    int nb[5];
    acdi_normal_d(P, s.psi, i, j, nx, ny, nb);
    const size_t k = cidx(i, j, P.g.Nx);
    s.nx[k] = nx.v;
    s.ny[k] = ny.v;
}

// One face of the ACDI flux: convective vel * phi_face and regularisation
// Gamma (eps d(phi)/dn - (1 - tanh^2(psi_f / 2 eps)) / 4 n_f).  Interior face:
// L, R the cells below / above it.  lam_c, lam_r: adjoints of the two fluxes.
__device__ void acdi_face_rev(const Params& P, const double* phi, const AdjScratch& s, int L, int R, double vel,
                              double h_i, double lc, double lr, bool xdir, double* lam_vel, AdjOut o) {
    Dn<7> pL = dseed<7>(phi[L], 0), pR = dseed<7>(phi[R], 1);
    Dn<7> sL = dseed<7>(s.psi[L], 2), sR = dseed<7>(s.psi[R], 3);
    Dn<7> nL = dseed<7>(xdir ? s.nx[L] : s.ny[L], 4), nR = dseed<7>(xdir ? s.nx[R] : s.ny[R], 5);
    Dn<7> u = dseed<7>(vel, 6);
    const double geff = P.md.pf_param[0], eps = P.md.pf_param[1];
    Dn<7> pf = 0.5 * pL + 0.5 * pR;
    Dn<7> cflux = u * pf;
    Dn<7> psf = 0.5 * sL + 0.5 * sR;
    // amp = (1 - tanh^2(psf / 2 eps)) / 4 as the forward flux has it, evaluated without
    // cancellation: in the saturated layers amp ~ min(phi, 1 - phi) multiplies a psi
    // slope ~ eps / min(phi, 1 - phi), and only accurate factors give their O(1) product
    Dn<7> amp = 0.25 * dsech2(psf / (2.0 * eps));
    Dn<7> nf = 0.5 * nL + 0.5 * nR;
    Dn<7> rflux = geff * (eps * ((pR - pL) * h_i) - amp * nf);
    Dn<7> F = lc * cflux + lr * rflux;
    atomicAdd(o.phi + L, F.d[0]);
    atomicAdd(o.phi + R, F.d[1]);
    atomicAdd(s.lpsi + L, F.d[2]);
    atomicAdd(s.lpsi + R, F.d[3]);
    atomicAdd((xdir ? s.lnx : s.lny) + L, F.d[4]);
    atomicAdd((xdir ? s.lnx : s.lny) + R, F.d[5]);
    atomicAdd(lam_vel, F.d[6]);
}

// Faces: x-face (i, j) for j < Ny, y-face (i, j) for i < Nx, over an (Nx+1) x (Ny+1) grid.
__global__ void k_adj_acdi_faces(Params P, AdjIn f, const double* __restrict__ lE, AdjScratch s, AdjOut o) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const bool px = P.g.px, py = P.g.py;
    // x-face i of row j: cells L = i-1, R = i (wrapped when periodic; face Nx is face 0)
    if (j < Ny && i <= Nx && !(px && i == Nx)) {
        const bool wall = !px && (i == 0 || i == Nx);
        const double vel = f.U[uidx(i, j, Nx)];
        double* lvel = o.U + uidx(i, j, Nx);
        if (wall) {
            const bool low = i == 0;
            const int I = (int)cidx(low ? 0 : Nx - 1, j, Nx);
            // flux appears as +c ihx in the cell above a low wall and -c ihx below a high one
            const double lc = (low ? 1.0 : -1.0) * P.g.ihx * lE[I];
            const SideD& sd = P.bphi.s[low ? LEFT : RIGHT];
            const bool dir = bdir(sd, j);
            const double pf = dir ? bval(sd, j) : f.phi[I];
            atomicAdd(lvel, lc * pf);
            if (!dir) atomicAdd(o.phi + I, lc * vel);
        } else {
            const int L = (int)cidx(wrapi(i - 1, Nx), j, Nx), R = (int)cidx(px ? wrapi(i, Nx) : i, j, Nx);
            const double lc = P.g.ihx * (lE[R] - lE[L]);
            acdi_face_rev(P, f.phi, s, L, R, vel, P.g.ihx, lc, -lc, true, lvel, o);
        }
    }
    if (i < Nx && j <= Ny && !(py && j == Ny)) {
        const bool wall = !py && (j == 0 || j == Ny);
        const double vel = f.V[vidx(i, j, Nx)];
        double* lvel = o.V + vidx(i, j, Nx);
        if (wall) {
            const bool low = j == 0;
            const int I = (int)cidx(i, low ? 0 : Ny - 1, Nx);
            const double lc = (low ? 1.0 : -1.0) * P.g.ihy * lE[I];
            const SideD& sd = P.bphi.s[low ? BOTTOM : TOP];
            const bool dir = bdir(sd, i);
            const double pf = dir ? bval(sd, i) : f.phi[I];
            atomicAdd(lvel, lc * pf);
            if (!dir) atomicAdd(o.phi + I, lc * vel);
        } else {
            const int L = (int)cidx(i, wrapi(j - 1, Ny), Nx), R = (int)cidx(i, py ? wrapi(j, Ny) : j, Nx);
            const double lc = P.g.ihy * (lE[R] - lE[L]);
            acdi_face_rev(P, f.phi, s, L, R, vel, P.g.ihy, lc, -lc, false, lvel, o);
        }
    }
}

// lam of psi from lam of the cell normals.
__global__ void k_adj_acdi_normals_rev(Params P, AdjScratch s) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= P.g.Nx || j >= P.g.Ny) return;
    const size_t k = cidx(i, j, P.g.Nx);
    const double ax = s.lnx[k], ay = s.lny[k];
    if (ax == 0.0 && ay == 0.0) return;
    Dn<5> nx, ny;
    int nb[5];
    acdi_normal_d(P, s.psi, i, j, nx, ny, nb);
    Dn<5> F = ax * nx + ay * ny;
#pragma unroll
    for (int q = 0; q < 5; ++q)
        if (nb[q] >= 0 && F.d[q] != 0.0) atomicAdd(s.lpsi + nb[q], F.d[q]);
}

// lam of phi from lam of psi = eps log((q + e) / (1 - q + e)), q = clamp(phi, 0, 1).
__global__ void k_adj_acdi_psi(Params P, const double* __restrict__ phi, AdjScratch s, double* lphi) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= P.g.Nx || j >= P.g.Ny) return;
    const size_t k = cidx(i, j, P.g.Nx);
    lphi[k] += s.lpsi[k] * acdi_dpsi(P.md, phi[k]);
}

// =====================================================================================
// Structure tensor (StructureTensor.jl:377-551; k_structure)
// =====================================================================================
// sigma log sigma of an SPD 2x2 tensor (a, d, b) (StructureTensor.jl:482-515):
// alpha sigma + beta I with eigenvalues m +- r, alpha = (g(m + r) - g(m - r)) / 2r and
// beta = (l+ g(m - r) - l- g(m + r)) / 2r for g(l) = l log l.  The forward's divided
// difference is exact in value up to rounding, but its derivative cancels two terms of
// size |dm| / r, which leaves an error of about eps m / r where the eigenvalues nearly
// coincide (1e-12 m < r << m: nearly isotropic tensors next to the reset region).  The
// reverse sweep therefore differentiates the same functions written in u = (r / m)^2,
// which is smooth in (a, d, b):
//   alpha = log m + F(u) + log(1 - u) / 2,  beta = -m (1 - u) F(u),
//   F(u) = atanh(sqrt u) / sqrt u = sum_k u^k / (2k + 1)  (the series below u = 1e-4).
// r <= 1e-12 scale keeps the forward's isotropic branch.
template <int K>
__device__ bool sigma_log_product_d(const Dn<K>& a, const Dn<K>& d, const Dn<K>& b, Dn<K>& oxx, Dn<K>& oyy,
                                    Dn<K>& oxy) {
    Dn<K> m = 0.5 * (a + d), del = 0.5 * (a - d);
    Dn<K> r = dhypot(del, b);
    Dn<K> lhi = m + r, llo = m - r;
    if (!(isfinite(llo.v) && isfinite(lhi.v) && llo.v > 0.0)) return false;
    const double scale = fmax(1.0, fabs(m.v));
    Dn<K> alpha, beta;
    if (r.v <= 1.0e-12 * scale) {
        alpha = dlog(m) + 1.0;
        beta = -m;
    } else {
        Dn<K> u = (del * del + b * b) / (m * m);
        Dn<K> F;
        if (u.v < 1.0e-4) {
            F = 1.0 + u * (1.0 / 3.0 + u * (1.0 / 5.0 + u * (1.0 / 7.0 + u * (1.0 / 9.0 + u * (1.0 / 11.0)))));
        } else {
            Dn<K> t = dsqrt(u);
            F = 0.5 * (dlog1p(t) - dlog1p(-t)) / t;
        }
        alpha = dlog(m) + F + 0.5 * dlog1p(-u);
        beta = -(m * (1.0 - u) * F);
    }
    oxx = alpha * a + beta;
    oyy = alpha * d + beta;
    oxy = alpha * b;
    return true;
}

// Upwind advection -div(v q) of one component at cell (i, j) (upwind_rhs<false>):
// lam of q (cells) and of the face velocities for the output adjoint lam.
__device__ void upwind_rev(const Params& P, const BCD& bc, const double* U, const double* V, const double* q, int i,
                           int j, double lam, double* lq, double* lU, double* lV) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    // flux(face) = vel * q_up; d(adv)/d(flux) = -/+ ihx
    auto face = [&](double lf, double vel, double* lvel, int up_cell, double up_val) {
        atomicAdd(lvel, lf * up_val);
        if (up_cell >= 0) atomicAdd(lq + up_cell, lf * vel);
    };
    auto inflow_is_data = [&](const SideD& s, double vel, bool low) {
        if (vel == 0.0) return false;
        const bool inflow = low ? vel > 0.0 : vel < 0.0;
        return inflow && s.type == EFSI_BC_DIRICHLET;
    };
    for (int side = 0; side < 2; ++side) {  // x faces i (side 0) and i + 1 (side 1)
        const int fidx = i + side;
        const double lf = (side ? -1.0 : 1.0) * P.g.ihx * lam;
        if (P.g.px) {
            const int fc = (fidx == Nx) ? 0 : fidx;
            const double u = U[uidx(fc, j, Nx)];
            const int c = u >= 0.0 ? (int)cidx(wrapi(fc - 1, Nx), j, Nx) : (int)cidx(fc, j, Nx);
            face(lf, u, lU + uidx(fc, j, Nx), c, q[c]);
        } else if (fidx == 0 || fidx == Nx) {
            const bool low = fidx == 0;
            const double u = U[uidx(fidx, j, Nx)];
            const int in = (int)cidx(low ? 0 : Nx - 1, j, Nx);
            const SideD& sd = bc.s[low ? LEFT : RIGHT];
            const bool data = inflow_is_data(sd, u, low);
            const bool use_b = low ? u >= 0.0 : u < 0.0;  // the upwind side is the boundary state
            if (use_b && data) face(lf, u, lU + uidx(fidx, j, Nx), -1, bval(sd, j));
            else face(lf, u, lU + uidx(fidx, j, Nx), in, q[in]);
        } else {
            const double u = U[uidx(fidx, j, Nx)];
            const int c = u >= 0.0 ? (int)cidx(fidx - 1, j, Nx) : (int)cidx(fidx, j, Nx);
            face(lf, u, lU + uidx(fidx, j, Nx), c, q[c]);
        }
    }
    for (int side = 0; side < 2; ++side) {  // y faces j (side 0) and j + 1 (side 1)
        const int fidx = j + side;
        const double lf = (side ? -1.0 : 1.0) * P.g.ihy * lam;
        if (P.g.py) {
            const int fc = (fidx == Ny) ? 0 : fidx;
            const double v = V[vidx(i, fc, Nx)];
            const int c = v >= 0.0 ? (int)cidx(i, wrapi(fc - 1, Ny), Nx) : (int)cidx(i, fc, Nx);
            face(lf, v, lV + vidx(i, fc, Nx), c, q[c]);
        } else if (fidx == 0 || fidx == Ny) {
            const bool low = fidx == 0;
            const double v = V[vidx(i, fidx, Nx)];
            const int in = (int)cidx(i, low ? 0 : Ny - 1, Nx);
            const SideD& sd = bc.s[low ? BOTTOM : TOP];
            const bool data = inflow_is_data(sd, v, low);
            const bool use_b = low ? v >= 0.0 : v < 0.0;
            if (use_b && data) face(lf, v, lV + vidx(i, fidx, Nx), -1, bval(sd, i));
            else face(lf, v, lV + vidx(i, fidx, Nx), in, q[in]);
        } else {
            const double v = V[vidx(i, fidx, Nx)];
            const int c = v >= 0.0 ? (int)cidx(i, fidx - 1, Nx) : (int)cidx(i, fidx, Nx);
            face(lf, v, lV + vidx(i, fidx, Nx), c, q[c]);
        }
    }
}

__global__ void k_adj_structure(Params P, AdjIn f, const double* __restrict__ lExx, const double* __restrict__ lEyy,
                                const double* __restrict__ lExy, AdjOut o, AdjParam par) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    const size_t k = cidx(i, j, Nx);
    const double lxx = lExx[k], lyy = lEyy[k], lxy = lExy[k];
    if (lxx == 0.0 && lyy == 0.0 && lxy == 0.0) return;
    const double* U = f.U;
    const double* V = f.V;
    const double ihx = P.g.ihx, ihy = P.g.ihy;
    auto Uc = [&](int r) { return 0.5 * U[uidx(i, r, Nx)] + 0.5 * U[uidx(i + 1, r, Nx)]; };
    auto Vc = [&](int c) { return 0.5 * V[vidx(c, j, Nx)] + 0.5 * V[vidx(c, j + 1, Nx)]; };
    auto wall_u = [&](const SideD& s, int a) { return 0.5 * bval(s, a) + 0.5 * bval(s, a + 1); };
    // velocity gradients (Operators.jl:474-583), the branches of k_structure
    double dudy, dvdx;
    int ybranch, xbranch;  // 0 centred (wrap when periodic), 1 low Dirichlet, 2 high Dirichlet, 3 constant
    if (P.g.py) { dudy = (Uc(wrapi(j + 1, Ny)) - Uc(wrapi(j - 1, Ny))) / (2.0 * P.g.hy); ybranch = 0; }
    else if (j == 0) {
        const SideD& s = P.bu.s[BOTTOM];
        if (s.type == EFSI_BC_DIRICHLET) { dudy = (Uc(0) - wall_u(s, i)) / (0.5 * P.g.hy); ybranch = 1; }
        else { dudy = -wall_u(s, i); ybranch = 3; }
    } else if (j == Ny - 1) {
        const SideD& s = P.bu.s[TOP];
        if (s.type == EFSI_BC_DIRICHLET) { dudy = (wall_u(s, i) - Uc(Ny - 1)) / (0.5 * P.g.hy); ybranch = 2; }
        else { dudy = wall_u(s, i); ybranch = 3; }
    } else { dudy = (Uc(j + 1) - Uc(j - 1)) / (2.0 * P.g.hy); ybranch = 0; }
    if (P.g.px) { dvdx = (Vc(wrapi(i + 1, Nx)) - Vc(wrapi(i - 1, Nx))) / (2.0 * P.g.hx); xbranch = 0; }
    else if (i == 0) {
        const SideD& s = P.bv.s[LEFT];
        if (s.type == EFSI_BC_DIRICHLET) { dvdx = (Vc(0) - wall_u(s, j)) / (0.5 * P.g.hx); xbranch = 1; }
        else { dvdx = -wall_u(s, j); xbranch = 3; }
    } else if (i == Nx - 1) {
        const SideD& s = P.bv.s[RIGHT];
        if (s.type == EFSI_BC_DIRICHLET) { dvdx = (wall_u(s, j) - Vc(Nx - 1)) / (0.5 * P.g.hx); xbranch = 2; }
        else { dvdx = wall_u(s, j); xbranch = 3; }
    } else { dvdx = (Vc(i + 1) - Vc(i - 1)) / (2.0 * P.g.hx); xbranch = 0; }
    const double dudx = (U[uidx(i + 1, j, Nx)] - U[uidx(i, j, Nx)]) * ihx;
    const double dvdy = (V[vidx(i, j + 1, Nx)] - V[vidx(i, j, Nx)]) * ihy;
    // local part: slots 0 dudx, 1 dvdy, 2 dudy, 3 dvdx, 4 sxx, 5 syy, 6 sxy, 7 phi
    Dn<8> a11 = dseed<8>(dudx, 0), a22 = dseed<8>(dvdy, 1), a12 = dseed<8>(dudy, 2), a21 = dseed<8>(dvdx, 3);
    Dn<8> sx = dseed<8>(f.sxx[k], 4), sy = dseed<8>(f.syy[k], 5), sc = dseed<8>(f.sxy[k], 6);
    Dn<8> divv = a11 + a22;
    Dn<8> exx = sx * divv + 2.0 * (a11 * sx + a12 * sc);
    Dn<8> eyy = sy * divv + 2.0 * (a21 * sc + a22 * sy);
    Dn<8> exy = sc * divv + (a21 * sx + a12 * sy + (a11 + a22) * sc);
    if (P.md.tensor_relaxation == EFSI_RELAX_MAXWELL) {
        const double rr = P.md.relaxation_rate;
        exx = exx + (-rr * (sx - 1.0));
        eyy = eyy + (-rr * (sy - 1.0));
        exy = exy + (-rr * sc);
    }
    if (P.nu.structure_extension == EFSI_EXT_GEOMETRIC) {
        Dn<8> ph = dseed<8>(f.phi[k], 7);
        Dn<8> kappa = P.nu.extension_rate * dpow(1.0 - dclamp01(ph), P.nu.extension_exponent);
        if (kappa.v != 0.0) {
            Dn<8> gx, gy, gxy;
            if (sigma_log_product_d(sx, sy, sc, gx, gy, gxy)) {
                exx = exx - kappa * gx;
                eyy = eyy - kappa * gy;
                exy = exy - kappa * gxy;
            }
        }
    }
    const Dn<8> F = lxx * exx + lyy * eyy + lxy * exy;
    atomicAdd(o.sxx + k, F.d[4]);
    atomicAdd(o.syy + k, F.d[5]);
    atomicAdd(o.sxy + k, F.d[6]);
    if (F.d[7] != 0.0) atomicAdd(o.phi + k, F.d[7]);
    // dudx, dvdy
    atomicAdd(o.U + uidx(i + 1, j, Nx), F.d[0] * ihx);
    atomicAdd(o.U + uidx(i, j, Nx), -F.d[0] * ihx);
    atomicAdd(o.V + vidx(i, j + 1, Nx), F.d[1] * ihy);
    atomicAdd(o.V + vidx(i, j, Nx), -F.d[1] * ihy);
    // dudy through Uc(r) = (U(i, r) + U(i+1, r)) / 2 and the wall data
    auto addUc = [&](int r, double g) {
        atomicAdd(o.U + uidx(i, r, Nx), 0.5 * g);
        atomicAdd(o.U + uidx(i + 1, r, Nx), 0.5 * g);
    };
    const double gy = F.d[2];
    if (ybranch == 0) {
        const double c = gy / (2.0 * P.g.hy);
        addUc(P.g.py ? wrapi(j + 1, Ny) : j + 1, c);
        addUc(P.g.py ? wrapi(j - 1, Ny) : j - 1, -c);
    } else if (ybranch == 1) {
        const double c = gy / (0.5 * P.g.hy);
        addUc(0, c);
        if (par.bu_bottom) { atomicAdd(par.bu_bottom + i, -0.5 * c); atomicAdd(par.bu_bottom + i + 1, -0.5 * c); }
    } else if (ybranch == 2) {
        const double c = gy / (0.5 * P.g.hy);
        addUc(Ny - 1, -c);
        if (par.bu_top) { atomicAdd(par.bu_top + i, 0.5 * c); atomicAdd(par.bu_top + i + 1, 0.5 * c); }
    }
    auto addVc = [&](int c, double g) {
        atomicAdd(o.V + vidx(c, j, Nx), 0.5 * g);
        atomicAdd(o.V + vidx(c, j + 1, Nx), 0.5 * g);
    };
    const double gx = F.d[3];
    if (xbranch == 0) {
        const double c = gx / (2.0 * P.g.hx);
        addVc(P.g.px ? wrapi(i + 1, Nx) : i + 1, c);
        addVc(P.g.px ? wrapi(i - 1, Nx) : i - 1, -c);
    } else if (xbranch == 1) {
        const double c = gx / (0.5 * P.g.hx);
        addVc(0, c);
        if (par.bv_left) { atomicAdd(par.bv_left + j, -0.5 * c); atomicAdd(par.bv_left + j + 1, -0.5 * c); }
    } else if (xbranch == 2) {
        const double c = gx / (0.5 * P.g.hx);
        addVc(Nx - 1, -c);
        if (par.bv_right) { atomicAdd(par.bv_right + j, 0.5 * c); atomicAdd(par.bv_right + j + 1, 0.5 * c); }
    }
    // advection of the three components
    if (lxx != 0.0) upwind_rev(P, P.bsxx, U, V, f.sxx, i, j, lxx, o.sxx, o.U, o.V);
    if (lyy != 0.0) upwind_rev(P, P.bsyy, U, V, f.syy, i, j, lyy, o.syy, o.U, o.V);
    if (lxy != 0.0) upwind_rev(P, P.bsxy, U, V, f.sxy, i, j, lxy, o.sxy, o.U, o.V);
}

// =====================================================================================
// Projection (Projection.jl:170-307), transposed
// =====================================================================================
// d(face gradient of q)/d(q of the cell above / below the face) for x-face i.
__device__ __forceinline__ void qgrad_coef_x(const Params& P, int i, int j, double& above, double& below) {
    const int Nx = P.g.Nx;
    above = below = 0.0;
    if (!P.g.px && (i == 0 || i == Nx)) {
        const SideD& s = P.bq.s[i == 0 ? LEFT : RIGHT];
        if (bdir(s, j)) {
            if (i == 0) above = 1.0 / (0.5 * P.g.hx);
            else below = -1.0 / (0.5 * P.g.hx);
        }
        return;
    }
    above = P.g.ihx;
    below = -P.g.ihx;
}
__device__ __forceinline__ void qgrad_coef_y(const Params& P, int i, int j, double& above, double& below) {
    const int Ny = P.g.Ny;
    above = below = 0.0;
    if (!P.g.py && (j == 0 || j == Ny)) {
        const SideD& s = P.bq.s[j == 0 ? BOTTOM : TOP];
        if (bdir(s, i)) {
            if (j == 0) above = 1.0 / (0.5 * P.g.hy);
            else below = -1.0 / (0.5 * P.g.hy);
        }
        return;
    }
    above = P.g.ihy;
    below = -P.g.ihy;
}

// omega = -Gq^T lam (the corrected velocity is U = Up - Gq q), written as the Poisson
// right-hand side b; its mean goes to ps->v[10] with a constant nullspace.  The periodic
// duplicate faces (x-face Nx, y-face Ny) carry the gradient of face 0.
__global__ void k_adj_proj_rhs(Params P, const double* __restrict__ lU, const double* __restrict__ lV, double* b,
                               int nullspace, ProjScal* ps, RedSlot rs) {
    __shared__ double sh[32];
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    double acc[1] = {0.0};
    if (i < Nx && j < Ny) {
        auto lu = [&](int f) {  // lam of x-face f, periodic duplicates folded onto face 0
            if (P.g.px && (f == 0 || f == Nx)) return lU[uidx(0, j, Nx)] + lU[uidx(Nx, j, Nx)];
            return lU[uidx(f, j, Nx)];
        };
        auto lv = [&](int f) {
            if (P.g.py && (f == 0 || f == Ny)) return lV[vidx(i, 0, Nx)] + lV[vidx(i, Ny, Nx)];
            return lV[vidx(i, f, Nx)];
        };
        double a, bl, om = 0.0;
        qgrad_coef_x(P, i, j, a, bl);       // left face: this cell is above
        om -= a * lu(i);
        qgrad_coef_x(P, i + 1, j, a, bl);   // right face: this cell is below
        om -= bl * lu(i + 1);
        qgrad_coef_y(P, i, j, a, bl);
        om -= a * lv(j);
        qgrad_coef_y(P, i, j + 1, a, bl);
        om -= bl * lv(j + 1);
        b[cidx(i, j, Nx)] = om;
        acc[0] = om;
    }
    double tot[1];
    if (grid_reduce<1>(acc, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        ps->v[10] = nullspace ? tot[0] / ((double)Nx * Ny) : 0.0;
        ps->v[3] = 0.0;
    }
}

// lam_pred = lam_U - area D^T y on the compact rows (y = x - mean); the periodic
// duplicate face Nx is the injected copy of face 0.
__global__ void k_adj_proj_finish(Params P, const double* __restrict__ x, const ProjScal* ps,
                                  const double* __restrict__ lU, const double* __restrict__ lV, double* lpu,
                                  double* lpv) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= Nx || j >= Ny) return;
    const double mean = ps->v[6];
    const double area = P.g.hx * P.g.hy;
    auto y = [&](int a, int c) { return x[cidx(a, c, Nx)] - mean; };
    // D Up at cell c = (Up(i+1) - Up(i)) ihx + ...: d/dUp(face f) = ihx (y(f-1) - y(f))
    double dx = (i > 0 ? y(i - 1, j) : 0.0) - y(i, j);
    double lu = lU[uidx(i, j, Nx)] - area * P.g.ihx * dx;
    if (P.g.px && i == 0) lu += lU[uidx(Nx, j, Nx)] - area * P.g.ihx * y(Nx - 1, j);
    double dy = (j > 0 ? y(i, j - 1) : 0.0) - y(i, j);
    double lv = lV[vidx(i, j, Nx)] - area * P.g.ihy * dy;
    if (P.g.py && j == 0) lv += lV[vidx(i, Ny, Nx)] - area * P.g.ihy * y(i, Ny - 1);
    lpu[cidx(i, j, Nx)] = lu;
    lpv[cidx(i, j, Nx)] = lv;
}

// Full MAC input (faces 0..Nx, 0..Ny): lam_in(f) = lam_U(f) - area ihx (y(f-1) - y(f)),
// y outside the grid taken as 0 (a face on the edge enters one cell's divergence).
__global__ void k_adj_proj_finish_full(Params P, const double* __restrict__ x, const ProjScal* ps,
                                       const double* __restrict__ lU, const double* __restrict__ lV, double* oU,
                                       double* oV) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const double mean = ps->v[6];
    const double area = P.g.hx * P.g.hy;
    auto y = [&](int a, int c) { return x[cidx(a, c, Nx)] - mean; };
    if (i <= Nx && j < Ny) {
        const double dx = (i > 0 ? y(i - 1, j) : 0.0) - (i < Nx ? y(i, j) : 0.0);
        oU[uidx(i, j, Nx)] = lU[uidx(i, j, Nx)] - area * P.g.ihx * dx;
    }
    if (i < Nx && j <= Ny) {
        const double dy = (j > 0 ? y(i, j - 1) : 0.0) - (j < Ny ? y(i, j) : 0.0);
        oV[vidx(i, j, Nx)] = lV[vidx(i, j, Nx)] - area * P.g.ihy * dy;
    }
}

// =====================================================================================
// Stage combinations (TimeIntegrationIMEX.jl:716-836), transposed
// =====================================================================================
__device__ __forceinline__ bool reset_at(const efsi_numerics& nu, double phi) {  // StructureTensor.jl:553-613
    if (nu.structure_extension == EFSI_EXT_IDENTITY_OUTSIDE) return phi < nu.extension_cutoff;
    if (nu.structure_extension == EFSI_EXT_GEOMETRIC) return nu.extension_cutoff > 0.0 && phi < nu.extension_cutoff;
    return false;
}

struct Hist {
    double* p[3];
};

__global__ void k_adj_vel_rhs(Params P, int s, double dt, const double* __restrict__ lru,
                              const double* __restrict__ lrv, double* luu, double* luv, Hist lEu, Hist lEv, Hist lIu,
                              Hist lIv, AdjParam par) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i >= Nx || j >= Ny) return;
    const size_t k = cidx(i, j, Nx);
    // the Dirichlet rows of the predictor take their data, not the right-hand side
    const bool ufix = !P.g.px && i == 0 && P.bu.s[LEFT].type == EFSI_BC_DIRICHLET;
    const bool vfix = !P.g.py && j == 0 && P.bv.s[BOTTOM].type == EFSI_BC_DIRICHLET;
    const double ru = ufix ? 0.0 : lru[k], rv = vfix ? 0.0 : lrv[k];
    luu[k] += ru;
    luv[k] += rv;
    for (int q = 0; q < s; ++q) {
        const double ae = a_AE[s][q], ai = a_AI[s][q];
        if (ae != 0.0) { lEu.p[q][k] += dt * ae * ru; lEv.p[q][k] += dt * ae * rv; }
        if (ai != 0.0) { lIu.p[q][k] += dt * ai * ru; lIv.p[q][k] += dt * ai * rv; }
    }
    if (P.md.viscosity == EFSI_VISC_NONE) return;
    // tangential wall data in the viscous boundary vector (visc_boundary, Operators.jl:1036-1080)
    const double alpha = dt * a_AI[s][s], mu = P.md.viscosity_fluid;
    if (!P.g.py) {
        const double w = mu / (P.g.hy * (0.5 * P.g.hy));
        if (j == 0 && P.bu.s[BOTTOM].type == EFSI_BC_DIRICHLET && par.bu_bottom) atomicAdd(par.bu_bottom + i, alpha * w * ru);
        if (j == Ny - 1 && P.bu.s[TOP].type == EFSI_BC_DIRICHLET && par.bu_top) atomicAdd(par.bu_top + i, alpha * w * ru);
    }
    if (!P.g.px) {
        const double w = mu / (P.g.hx * (0.5 * P.g.hx));
        if (i == 0 && P.bv.s[LEFT].type == EFSI_BC_DIRICHLET && par.bv_left) atomicAdd(par.bv_left + j, alpha * w * rv);
        if (i == Nx - 1 && P.bv.s[RIGHT].type == EFSI_BC_DIRICHLET && par.bv_right) atomicAdd(par.bv_right + j, alpha * w * rv);
    }
}

__global__ void k_adj_combine(Params P, int s, double dt, const double* __restrict__ phis,
                              const double* __restrict__ lphi, const double* __restrict__ lsx,
                              const double* __restrict__ lsy, const double* __restrict__ lsc, double* lphin,
                              double* lsxn, double* lsyn, double* lscn, Hist lEphi, Hist lExx, Hist lEyy, Hist lExy) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= P.g.Nx || j >= P.g.Ny) return;
    const size_t k = cidx(i, j, P.g.Nx);
    const bool keep = !reset_at(P.nu, phis[k]);
    const double p = lphi[k], a = keep ? lsx[k] : 0.0, d = keep ? lsy[k] : 0.0, c = keep ? lsc[k] : 0.0;
    lphin[k] += p;
    lsxn[k] += a;
    lsyn[k] += d;
    lscn[k] += c;
    for (int q = 0; q < s; ++q) {
        const double ae = a_AE[s][q];
        if (ae == 0.0) continue;
        const double w = dt * ae;
        lEphi.p[q][k] += w * p;
        lExx.p[q][k] += w * a;
        lEyy.p[q][k] += w * d;
        lExy.p[q][k] += w * c;
    }
}

__global__ void k_adj_step_start(Params P, const double* __restrict__ phin, const double* __restrict__ lU0,
                                 const double* __restrict__ lV0, const double* __restrict__ luu,
                                 const double* __restrict__ luv, const double* __restrict__ lphi0,
                                 const double* __restrict__ lphin, const double* __restrict__ lsx0,
                                 const double* __restrict__ lsy0, const double* __restrict__ lsc0,
                                 const double* __restrict__ lsxn, const double* __restrict__ lsyn,
                                 const double* __restrict__ lscn, double* oU, double* oV, double* ophi, double* osx,
                                 double* osy, double* osc) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    if (i <= Nx && j < Ny) oU[uidx(i, j, Nx)] = lU0[uidx(i, j, Nx)] + (i < Nx ? luu[cidx(i, j, Nx)] : 0.0);
    if (i < Nx && j <= Ny) oV[vidx(i, j, Nx)] = lV0[vidx(i, j, Nx)] + (j < Ny ? luv[cidx(i, j, Nx)] : 0.0);
    if (i < Nx && j < Ny) {
        const size_t k = cidx(i, j, Nx);
        ophi[k] = lphi0[k] + lphin[k];
        const bool keep = !reset_at(P.nu, phin[k]);
        osx[k] = keep ? lsx0[k] + lsxn[k] : 0.0;
        osy[k] = keep ? lsy0[k] + lsyn[k] : 0.0;
        osc[k] = keep ? lsc0[k] + lscn[k] : 0.0;
    }
}

__global__ void k_adj_reset_sigma(Params P, const double* __restrict__ phi, const double* __restrict__ sx,
                                  const double* __restrict__ sy, const double* __restrict__ sc, double* ox,
                                  double* oy, double* oc) {
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= P.g.Nx || j >= P.g.Ny) return;
    const size_t k = cidx(i, j, P.g.Nx);
    const bool r = reset_at(P.nu, phi[k]);
    ox[k] = r ? 1.0 : sx[k];
    oy[k] = r ? 1.0 : sy[k];
    oc[k] = r ? 0.0 : sc[k];
}

__global__ void k_adj_record(int nu, int nv, int nc, const int* __restrict__ counter, size_t stride, size_t off,
                             const double* __restrict__ U, const double* __restrict__ V,
                             const double* __restrict__ phi, const double* __restrict__ sx,
                             const double* __restrict__ sy, const double* __restrict__ sc, double* tape) {
    double* base = tape + (size_t)(*counter) * stride + off;
    const int n = max(nu, max(nv, nc));
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        if (k < nu && U) base[k] = U[k];
        if (k < nv && V) base[nu + k] = V[k];
        if (k < nc) {
            if (phi) base[nu + nv + k] = phi[k];
            if (sx) base[nu + nv + nc + k] = sx[k];
            if (sy) base[nu + nv + 2 * (size_t)nc + k] = sy[k];
            if (sc) base[nu + nv + 3 * (size_t)nc + k] = sc[k];
        }
    }
}

}  // namespace

// =========================================================================================
// host side
// =========================================================================================
const char* adjoint_unsupported(const Params& P, bool resource, bool growth) {
    const efsi_models& m = P.md;
    if (resource || growth) return "the adjoint does not differentiate growth or resource transport";
    if (m.phase_field_method != EFSI_PF_ACDI) return "the adjoint differentiates the ACDI phase-field method only";
    if (m.pf_option) return "the adjoint does not differentiate the dynamic ACDI mobility";
    if (m.viscosity != EFSI_VISC_NONE && m.viscosity != EFSI_VISC_CONSTANT)
        return "the adjoint differentiates constant (or no) viscosity only";
    if (m.capillarity != EFSI_CAP_NONE) return "the adjoint does not differentiate capillarity";
    return "";
}

Params homogeneous(const Params& P) {
    Params H = P;
    BCD* all[8] = {&H.bu, &H.bv, &H.bq, &H.bphi, &H.bc, &H.bsxx, &H.bsyy, &H.bsxy};
    for (BCD* b : all)
        for (SideD& s : b->s) { s.val = nullptr; s.neu = nullptr; }
    for (double& v : H.psi_bc) v = 0.0;
    return H;
}

void adj_tendencies(const Params& P, const AdjIn& f, const AdjTend& lt, const AdjOut& out, const AdjParam& par,
                    const AdjScratch& sc, DevStatus* st, cudaStream_t s) {
    const dim3 g = grid2(P.g.Nx, P.g.Ny), gf = grid2(P.g.Nx + 1, P.g.Ny + 1), b(BX, BY);
    const size_t N = (size_t)P.g.Nx * P.g.Ny;
    Lam L{};
    L.p[T_U] = out.U; L.p[T_V] = out.V; L.p[T_PHI] = out.phi;
    L.p[T_SXX] = out.sxx; L.p[T_SYY] = out.syy; L.p[T_SXY] = out.sxy;
    L.p[T_BUB] = par.bu_bottom; L.p[T_BUT] = par.bu_top; L.p[T_BVL] = par.bv_left; L.p[T_BVR] = par.bv_right;
    L.p[T_TXX] = sc.ltxx; L.p[T_TYY] = sc.ltyy; L.p[T_TXY] = sc.ltxy;
    // momentum forcing: convection into U, V; stress divergence into the cell stresses
    const int elastic = P.md.elastic_stress == EFSI_ELASTIC_LINEAR;
    if (elastic) {
        cudaMemsetAsync(sc.ltxx, 0, N * sizeof(double), s);
        cudaMemsetAsync(sc.ltyy, 0, N * sizeof(double), s);
        cudaMemsetAsync(sc.ltxy, 0, N * sizeof(double), s);
    }
    k_adj_momentum<<<g, b, 0, s>>>(P, f, lt.Eu, lt.Ev, L, elastic, st);
    if (elastic) k_adj_tau<<<g, b, 0, s>>>(P, f, sc.ltxx, sc.ltyy, sc.ltxy, out, par.G);
    // viscous operator history I_uv
    if (P.md.viscosity != EFSI_VISC_NONE) k_adj_visc<<<g, b, 0, s>>>(P, f, lt.Iu, lt.Iv, L, st);
    // ACDI phase field: psi -> cell normals -> face fluxes, reversed link by link
    k_adj_acdi_cells<<<g, b, 0, s>>>(P, f.phi, sc);
    k_adj_acdi_normals<<<g, b, 0, s>>>(P, sc);
    k_adj_acdi_faces<<<gf, b, 0, s>>>(P, f, lt.Ephi, sc, out);
    k_adj_acdi_normals_rev<<<g, b, 0, s>>>(P, sc);
    k_adj_acdi_psi<<<g, b, 0, s>>>(P, f.phi, sc, out.phi);
    // structure tensor
    k_adj_structure<<<g, b, 0, s>>>(P, f, lt.Exx, lt.Eyy, lt.Exy, out, par);
}

void adj_proj_rhs(const Params& P, const Projection& pj, const double* lamU, const double* lamV, ProjScal* ps,
                  const RedSlot& rs, cudaStream_t s) {
    k_adj_proj_rhs<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, lamU, lamV, pj.b, pj.nullspace ? 1 : 0, ps, rs);
}
void adj_proj_finish(const Params& P, const Projection& pj, const double* lamU, const double* lamV,
                     const ProjScal* ps, double* lam_pu, double* lam_pv, cudaStream_t s) {
    k_adj_proj_finish<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, pj.x, ps, lamU, lamV, lam_pu, lam_pv);
}

void adj_proj_finish_full(const Params& P, const Projection& pj, const double* lamU, const double* lamV,
                          const ProjScal* ps, double* lam_U_in, double* lam_V_in, cudaStream_t s) {
    k_adj_proj_finish_full<<<grid2(P.g.Nx + 1, P.g.Ny + 1), dim3(BX, BY), 0, s>>>(P, pj.x, ps, lamU, lamV, lam_U_in,
                                                                                  lam_V_in);
}

void adj_velocity_rhs(const Params& P, int stage, double dt, const double* lr_u, const double* lr_v,
                      double* luvn_u, double* luvn_v, double* const* lEu, double* const* lEv, double* const* lIu,
                      double* const* lIv, const AdjParam& par, cudaStream_t s) {
    Hist a{}, b{}, c{}, d{};
    for (int q = 0; q < 3; ++q) { a.p[q] = lEu[q]; b.p[q] = lEv[q]; c.p[q] = lIu[q]; d.p[q] = lIv[q]; }
    k_adj_vel_rhs<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, stage, dt, lr_u, lr_v, luvn_u, luvn_v, a, b, c,
                                                                 d, par);
}

void adj_combine(const Params& P, int stage, double dt, const double* phis, const double* lphi,
                 const double* lsxx, const double* lsyy, const double* lsxy, double* lphin, double* lsxn,
                 double* lsyn, double* lsxyn, double* const* lEphi, double* const* lExx, double* const* lEyy,
                 double* const* lExy, cudaStream_t s) {
    Hist a{}, b{}, c{}, d{};
    for (int q = 0; q < 3; ++q) { a.p[q] = lEphi[q]; b.p[q] = lExx[q]; c.p[q] = lEyy[q]; d.p[q] = lExy[q]; }
    k_adj_combine<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, stage, dt, phis, lphi, lsxx, lsyy, lsxy, lphin,
                                                                 lsxn, lsyn, lsxyn, a, b, c, d);
}

void adj_step_start(const Params& P, const double* phin, const double* lU0, const double* lV0,
                    const double* luvn_u, const double* luvn_v, const double* lphi0, const double* lphin,
                    const double* lsx0, const double* lsy0, const double* lsxy0, const double* lsxn,
                    const double* lsyn, const double* lsxyn, double* oU, double* oV, double* ophi, double* osxx,
                    double* osyy, double* osxy, cudaStream_t s) {
    k_adj_step_start<<<grid2(P.g.Nx + 1, P.g.Ny + 1), dim3(BX, BY), 0, s>>>(
        P, phin, lU0, lV0, luvn_u, luvn_v, lphi0, lphin, lsx0, lsy0, lsxy0, lsxn, lsyn, lsxyn, oU, oV, ophi, osxx,
        osyy, osxy);
}

void adj_reset_sigma(const Params& P, const double* phi, const double* sxx, const double* syy, const double* sxy,
                     double* oxx, double* oyy, double* oxy, cudaStream_t s) {
    k_adj_reset_sigma<<<grid2(P.g.Nx, P.g.Ny), dim3(BX, BY), 0, s>>>(P, phi, sxx, syy, sxy, oxx, oyy, oxy);
}

void adj_record(const Params& P, const int* counter, size_t slot_stride, size_t offset, const double* U,
                const double* V, const double* phi, const double* sxx, const double* syy, const double* sxy,
                double* tape, cudaStream_t s) {
    const int Nx = P.g.Nx, Ny = P.g.Ny;
    const int nu = (Nx + 1) * Ny, nv = Nx * (Ny + 1), nc = Nx * Ny;
    const int n = std::max(nu, nv);
    k_adj_record<<<std::min((n + 255) / 256, 4 * std::max(P.nsm, 1)), 256, 0, s>>>(nu, nv, nc, counter, slot_stride,
                                                                                 offset, U, V, phi, sxx, syy, sxy,
                                                                                 tape);
}

}  // namespace efsi
