// efsi_api.cu — C-ABI of the B200 IMEX step (include/efsi.h): context creation,
// device buffers, the four-stage orchestration of TimeIntegrationIMEX.jl:1152-1256
// and the operator-level entry points.
//
// Orchestration: one CUDA stream per handle.  The whole step is captured once as a
// CUDA graph; every Krylov solve keeps its scalars on the device and becomes a
// conditional WHILE node whose body (two iterations) clears the loop flag when the
// residual test passes, so a step is one graph launch and a batch of steps needs
// one host synchronisation.  (t, dt) come from a device array indexed by a step
// counter, so the same graph serves every step.  When a launch site is being timed
// (or efsi_set_step_mode selects EFSI_STEP_HOST) the step is enqueued from the host instead, with the solves
// in batches sized from the previous solve's iteration count.  Device-side errors
// (the Julia exceptions of the reference) are raised into a status word and
// reported after the step; a failing step leaves the state untouched.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "efsi_adjoint.cuh"
#include "efsi_diag.cuh"
#include "efsi_kernels.cuh"
#include "efsi_solvers.cuh"

using namespace efsi;

namespace {

struct DevBlock {
    DevStatus st;
    CGScal cg_visc, cg_diff, cg_proj;
    ProjScal ps;
    double report[6];
    long long nonspd;
    double max_constraint;
    double max_trace;
    double gamma_dyn;
    double t, dt;         // current step (read by the kernels: a captured graph serves every dt)
    int counter;          // steps completed in the current batch
    int first_fail;       // batch index of the first failing step, -1 if none
    int iters[3][4];      // CG iterations of the current step: [projection|velocity|resource][stage]
};

// Per-step record written on the device at the end of every step.
struct StepRec {
    double v[7];          // StepReport (constraint, trace, min/max phi, min c, min eig, |det-1|)
    long long nonspd;
    int iters[3][4];
};
constexpr int kMaxBatch = 1024;  // steps per device batch (efsi_step_n is chunked)

struct Err {
    int code;
    std::string msg;
};

thread_local std::string g_create_error;

const char* bc_name(int t) {
    switch (t) {
        case EFSI_BC_PERIODIC: return "Periodic";
        case EFSI_BC_DIRICHLET: return "Dirichlet";
        case EFSI_BC_NEUMANN: return "Neumann";
        case EFSI_BC_MIXED: return "MixedBoundary";
        case EFSI_BC_ADVECTIVE_OUTFLOW: return "AdvectiveOutflow";
    }
    return "unknown";
}

}  // namespace

struct efsi_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    Params P{};
    int Nx = 0, Ny = 0;
    size_t nc = 0, nu = 0, nv = 0;
    std::vector<void*> allocs;
    std::string err;
    efsi_stats stats{};
    bool visc = false, diff = false, growth = false, resource = false;
    Err step_block{EFSI_OK, ""};  // why this configuration cannot step (empty: it can)
    // state and correction
    double *U, *V, *phi, *c, *sxx, *syy, *sxy, *q;
    // stage buffers
    double *Us, *Vs, *phis, *cs, *sxs, *sys, *sxys, *sxn, *syn, *sxyn, *G;
    double *Eu[3], *Ev[3], *Iu[3], *Iv[3], *Ephi[3], *Exx[3], *Eyy[3], *Exy[3], *Ec[3], *Ic[3];
    double *rhs_u, *rhs_v, *rhs_c;
    double *kappa, *cap_a, *cap_b;
    ViscSolve vs{};
    ViscMixed vm{};     // precision form: FP32 vectors of the refined viscous solve
    bool mixed = false;
    ScalarSolve ds{};
    Projection pj{};
    DevBlock* dev = nullptr;   // device scalars
    DevBlock* host = nullptr;  // pinned mirror
    int* done_pinned = nullptr;
    RedSlot slot[8];
    // driver diagnostics: reduction slots sized for 32 values, device totals, pinned copy
    static constexpr int kDiagBlocks = 1024;
    RedSlot dslot[3];
    double* diag_dev = nullptr;
    double* diag_pinned = nullptr;
    // solver batch predictions (host-driven mode)
    int pred[3] = {4, 4, 4};
    long long launches = 0;
    // step graphs: the whole IMEX step captured once, CG loops as WHILE nodes; slot 1 is
    // the same step with the tape records of the differentiation form
    cudaStream_t stream2 = nullptr;
    bool use_graph = true, capturing = false;
    struct Loop { int kind, stage, kernels_per_body, iters_per_body; };
    struct GraphSlot {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        long long fixed_launches = 0;
        std::vector<Loop> loops;
    };
    GraphSlot gs[2];
    // differentiation form: the state every `adj_every` steps of the last
    // efsi_forward_checkpointed call, the tape of one recomputed segment, and the
    // adjoint buffers (allocated on first use)
    bool recording = false;
    int adj_n = 0, adj_every = 0, adj_ckpt_cap = 0, adj_tape_cap = 0;
    double adj_t0 = 0.0;
    std::vector<double> adj_dts;
    double* ckpt = nullptr;         // adj_ckpt_cap slots of ckpt_stride()
    double* tape = nullptr;         // adj_tape_cap slots of tape_stride()
    double* adj = nullptr;          // adjoint buffers, see adjoint_buffers()
    size_t adj_words = 0;
    struct AdjBufs {
        double *lU, *lV, *lphi, *lsxx, *lsyy, *lsxy;     // adjoint of the state (in and out of a reverse step)
        double *sU, *sV, *sphi, *ssxx, *ssyy, *ssxy;     // adjoint of one stage's fields
        double *acc;                                     // start of the block cleared per reverse step:
        double *luu, *luv, *lphin, *lsxn, *lsyn, *lscn;  //   adjoint of uv_n, phi_n, sigma_n'
        double *lEu[3], *lEv[3], *lIu[3], *lIv[3], *lEphi[3], *lExx[3], *lEyy[3], *lExy[3];  //   of histories
        size_t acc_words;
        double *lpu, *lpv;                               // adjoint of the predictor (compact)
        double *zU, *zV, *zq;                            // zeros: starts of the adjoint solves
        double *s0x, *s0y, *s0c;                         // sigma_n' of the step being reversed
        double *final_state;                             // the state after the forward sweep (restored)
        AdjScratch sc;
        double *bub, *but, *bvl, *bvr, *G;               // parameter adjoints
    } ab{};
    size_t block_words() const { return nu + nv + 4 * nc; }            // U, V, phi, sigma x3
    size_t tape_stride() const { return 3 * block_words() + nc; }      // start, stage 1, stage 2, phi_3
    size_t ckpt_stride() const { return nu + nv + 6 * nc; }            // U, V, phi, c, sigma x3, q
    double* times_dev = nullptr;    // (t, dt) per step of a batch
    double* times_pinned = nullptr;
    StepRec* hist_dev = nullptr;
    StepRec* hist_pinned = nullptr;
    // CUDA-event timing: whole calls and one selectable launch site
    cudaEvent_t call_ev[2] = {nullptr, nullptr};
    int timed_site = EFSI_SITE_NONE;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> site_ev;
    size_t site_used = 0;
    double site_bytes_pending = 0.0;
    double step_bytes_pending = 0.0;  // algorithmic bytes of every site launch (host-driven)

    template <class T>
    T* dalloc(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess)
            throw Err{EFSI_CUDA, "cudaMalloc failed"};
        cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
        allocs.push_back(p);
        return static_cast<T*>(p);
    }
    ~efsi_handle() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& e : site_ev) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
        for (cudaEvent_t e : call_ev) if (e) cudaEventDestroy(e);
        for (void* p : allocs) cudaFree(p);
        for (double* p : {ckpt, tape, adj}) if (p) cudaFree(p);
        for (GraphSlot& g : gs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            if (g.graph) cudaGraphDestroy(g.graph);
        }
        if (host) cudaFreeHost(host);
        if (done_pinned) cudaFreeHost(done_pinned);
        if (times_pinned) cudaFreeHost(times_pinned);
        if (diag_pinned) cudaFreeHost(diag_pinned);
        if (hist_pinned) cudaFreeHost(hist_pinned);
        if (stream2) cudaStreamDestroy(stream2);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Err{EFSI_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

void reset_call_stats(efsi_handle* h) {
    std::memset(h->stats.projection_iterations, 0, sizeof(h->stats.projection_iterations));
    std::memset(h->stats.velocity_iterations, 0, sizeof(h->stats.velocity_iterations));
    std::memset(h->stats.resource_iterations, 0, sizeof(h->stats.resource_iterations));
    h->stats.kernel_launches = 0;
    h->stats.device_ms = 0.0;
    h->launches = 0;
}

// Bracket a launch site with CUDA events when it is the timed one.
template <class F>
void site(efsi_handle* h, int which, double bytes, F&& f) {
    if (!h->capturing) h->step_bytes_pending += bytes;
    if (h->capturing || h->timed_site != which) { f(); return; }
    if (h->site_used == h->site_ev.size()) {
        cudaEvent_t a, b;
        check_cuda(cudaEventCreate(&a), "event");
        check_cuda(cudaEventCreate(&b), "event");
        h->site_ev.emplace_back(a, b);
    }
    auto& e = h->site_ev[h->site_used++];
    check_cuda(cudaEventRecord(e.first, h->stream), "event");
    f();
    check_cuda(cudaEventRecord(e.second, h->stream), "event");
    h->site_bytes_pending += bytes;
}

// After the stream is idle: fold the recorded site events into the statistics.
void collect_site_events(efsi_handle* h) {
    for (size_t k = 0; k < h->site_used; ++k) {
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, h->site_ev[k].first, h->site_ev[k].second), "event");
        h->stats.site_ms += ms;
        h->stats.site_launches += 1;
    }
    h->stats.site_bytes += h->site_bytes_pending;
    h->stats.step_bytes += h->step_bytes_pending;
    h->site_used = 0;
    h->site_bytes_pending = 0.0;
    h->step_bytes_pending = 0.0;
}

void call_begin(efsi_handle* h) { check_cuda(cudaEventRecord(h->call_ev[0], h->stream), "event"); }
void call_end(efsi_handle* h) {
    check_cuda(cudaEventRecord(h->call_ev[1], h->stream), "event");
    check_cuda(cudaEventSynchronize(h->call_ev[1]), "event");
    float ms = 0.f;
    check_cuda(cudaEventElapsedTime(&ms, h->call_ev[0], h->call_ev[1]), "event");
    h->stats.device_ms = ms;
    collect_site_events(h);
}

// ---------------------------------------------------------------------------------------
// configuration validation
// ---------------------------------------------------------------------------------------
double uniform_spacing(const double* a, int n, double h, const char* name) {
    if (!a) throw Err{EFSI_ARG, std::string("mesh metric ") + name + " missing"};
    for (int k = 0; k < n; ++k)
        if (!(std::fabs(a[k] - h) <= 1e-12 * std::fabs(h)))
            throw Err{EFSI_UNSUPPORTED, std::string("the device step requires uniform spacing; ") + name +
                                            " is stretched (MeshGeneration.jl stretchings are not supported)"};
    return h;
}

void upload_side(efsi_handle* h, const efsi_bc_side& in, int need, SideD& out, const char* what) {
    out.type = in.type;
    out.val = nullptr; out.neu = nullptr; out.mask = nullptr;
    if (in.type < EFSI_BC_PERIODIC || in.type > EFSI_BC_ADVECTIVE_OUTFLOW)
        throw Err{EFSI_ARG, std::string(what) + ": unknown boundary type"};
    if (in.type == EFSI_BC_PERIODIC) return;
    if (in.n < need) throw Err{EFSI_DIM, std::string(what) + ": boundary data shorter than the side"};
    if (in.value) {
        double* d = h->dalloc<double>(in.n);
        check_cuda(cudaMemcpy(d, in.value, sizeof(double) * in.n, cudaMemcpyHostToDevice), "bc upload");
        out.val = d;
    }
    if (in.type == EFSI_BC_MIXED) {
        if (in.neumann) {
            double* d = h->dalloc<double>(in.n);
            check_cuda(cudaMemcpy(d, in.neumann, sizeof(double) * in.n, cudaMemcpyHostToDevice), "bc upload");
            out.neu = d;
        }
        uint8_t* m = h->dalloc<uint8_t>(in.n);
        if (in.mask) check_cuda(cudaMemcpy(m, in.mask, in.n, cudaMemcpyHostToDevice), "bc upload");
        out.mask = m;
    }
}

void upload_bcs(efsi_handle* h, const efsi_bc_setup& in, int n_lr, int n_bt, BCD& out, const char* name) {
    const efsi_bc_side* s[4] = {&in.left, &in.right, &in.bottom, &in.top};
    for (int k = 0; k < 4; ++k) upload_side(h, *s[k], k < 2 ? n_lr : n_bt, out.s[k], name);
    if ((in.left.type == EFSI_BC_PERIODIC) != (in.right.type == EFSI_BC_PERIODIC))
        throw Err{EFSI_ARG, std::string(name) + ": periodic boundaries in the x-direction must be specified as an opposing pair."};
    if ((in.bottom.type == EFSI_BC_PERIODIC) != (in.top.type == EFSI_BC_PERIODIC))
        throw Err{EFSI_ARG, std::string(name) + ": periodic boundaries in the y-direction must be specified as an opposing pair."};
}

bool side_has_dirichlet(const efsi_bc_side& s) {
    if (s.type == EFSI_BC_DIRICHLET) return true;
    if (s.type == EFSI_BC_MIXED && s.mask)
        for (int k = 0; k < s.n; ++k)
            if (s.mask[k]) return true;
    return false;
}

// Requirements that only integrate_step! enforces; an empty message means the
// configuration can step.
Err step_requirements(const efsi_config& cfg) {
    if (!cfg.mesh.periodic_x && cfg.bc_U.right.type != EFSI_BC_DIRICHLET)
        return {EFSI_ARG, "The compact predictor currently requires a Dirichlet or Periodic U-right boundary."};
    if (!cfg.mesh.periodic_y && cfg.bc_V.top.type != EFSI_BC_DIRICHLET)
        return {EFSI_ARG, "The compact predictor currently requires a Dirichlet or Periodic V-top boundary."};
    auto dn = [](int t) { return t == EFSI_BC_DIRICHLET || t == EFSI_BC_NEUMANN; };
    if (!cfg.mesh.periodic_y && !(dn(cfg.bc_U.bottom.type) && dn(cfg.bc_U.top.type)))
        return {EFSI_ARG, "Unsupported U-bottom/top boundary for du/dy: Dirichlet or Neumann required."};
    if (!cfg.mesh.periodic_x && !(dn(cfg.bc_V.left.type) && dn(cfg.bc_V.right.type)))
        return {EFSI_ARG, "Unsupported V-left/right boundary for dv/dx: Dirichlet or Neumann required."};
    return {EFSI_OK, ""};
}

void validate_models(const efsi_config& cfg) {
    const efsi_models& md = cfg.models;
    const efsi_bc_setup* all[8] = {&cfg.bc_U, &cfg.bc_V, &cfg.bc_correction, &cfg.bc_phi, &cfg.bc_resource,
                                   &cfg.bc_sigma_xx, &cfg.bc_sigma_yy, &cfg.bc_sigma_xy};
    const char* names[8] = {"U", "V", "correction", "phi", "resource", "sigma_xx", "sigma_yy", "sigma_xy"};
    for (int k = 0; k < 8; ++k) {  // TimeIntegrationIMEX.jl:447-466
        if ((all[k]->left.type == EFSI_BC_PERIODIC) != (cfg.mesh.periodic_x != 0))
            throw Err{EFSI_ARG, std::string(names[k]) + " boundary conditions do not match MeshMetrics periodicity in x."};
        if ((all[k]->bottom.type == EFSI_BC_PERIODIC) != (cfg.mesh.periodic_y != 0))
            throw Err{EFSI_ARG, std::string(names[k]) + " boundary conditions do not match MeshMetrics periodicity in y."};
    }
    if (md.viscosity != EFSI_VISC_NONE) {  // Operators.jl:89-105
        const efsi_bc_side* vs[8] = {&cfg.bc_U.left, &cfg.bc_U.right, &cfg.bc_U.bottom, &cfg.bc_U.top,
                                     &cfg.bc_V.left, &cfg.bc_V.right, &cfg.bc_V.bottom, &cfg.bc_V.top};
        const char* vn[8] = {"U-left", "U-right", "U-bottom", "U-top", "V-left", "V-right", "V-bottom", "V-top"};
        for (int k = 0; k < 8; ++k)
            if (vs[k]->type != EFSI_BC_DIRICHLET && vs[k]->type != EFSI_BC_PERIODIC)
                throw Err{EFSI_ARG, std::string(vn[k]) + " uses " + bc_name(vs[k]->type) +
                                        ". The current compact viscous operator supports Dirichlet or Periodic velocity boundaries."};
    }
    // Step-only requirements (compact predictor injection, TimeIntegrationIMEX.jl:554-576;
    // tangential velocity data of velocity_gradient / convection, Operators.jl:503-579,
    // MomentumTransport.jl:89-102) are reported by integrate_step, as in the reference.
    // Phase-field boundary rules (PhaseFieldMethods.jl:174-196, :493-529, :352-375).
    const efsi_bc_side* ph[4] = {&cfg.bc_phi.left, &cfg.bc_phi.right, &cfg.bc_phi.bottom, &cfg.bc_phi.top};
    const double tiny = 100 * 2.220446049250313e-16;
    if (md.phase_field_method == EFSI_PF_ACDI || md.phase_field_method == EFSI_PF_UWCDI) {
        for (const efsi_bc_side* s : ph) {
            if (s->type == EFSI_BC_NEUMANN && s->value)
                for (int k = 0; k < s->n; ++k)
                    if (std::fabs(s->value[k]) > tiny)
                        throw Err{EFSI_ARG, "Only homogeneous Neumann phase boundaries are supported by the ACDI/UWCDI operators."};
            if (s->type == EFSI_BC_MIXED && s->neumann)
                for (int k = 0; k < s->n; ++k)
                    if (!(s->mask && s->mask[k]) && std::fabs(s->neumann[k]) > tiny)
                        throw Err{EFSI_ARG, "Only homogeneous-Neumann mixed phase faces are supported here."};
        }
    }
    if (md.phase_field_method == EFSI_PF_ACDI) {
        for (const efsi_bc_side* s : ph) {
            if (s->type == EFSI_BC_PERIODIC || s->type == EFSI_BC_NEUMANN) continue;
            if (s->type == EFSI_BC_DIRICHLET) {
                for (int k = 1; k < s->n; ++k)
                    if (s->value && s->value[k] != s->value[0])
                        throw Err{EFSI_ARG, "ACDI psi transformation currently requires scalar Dirichlet phase data."};
                continue;
            }
            throw Err{EFSI_ARG, "ACDI psi geometry supports Periodic, homogeneous Neumann, or scalar Dirichlet phase boundaries."};
        }
    }
    if (md.phase_field_method == EFSI_PF_UWCDI && md.pf_option == EFSI_NORMALS_SMOOTHED9) {
        for (const efsi_bc_side* s : ph) {
            if (s->type == EFSI_BC_PERIODIC) continue;
            if (s->type == EFSI_BC_NEUMANN && !(s->value && std::fabs(s->value[0]) > tiny)) continue;
            throw Err{EFSI_ARG, "smoothed9 normal reconstruction requires homogeneous Neumann or periodic phase boundaries."};
        }
    }
    if (md.phase_field_method < EFSI_PF_UPWIND || md.phase_field_method > EFSI_PF_UWCDI)
        throw Err{EFSI_ARG, "phase_field_method must be an AbstractPhaseFieldMethod."};
}

// ---------------------------------------------------------------------------------------
// multigrid hierarchy and the dense coarse inverse
// ---------------------------------------------------------------------------------------
struct HostLevel {
    int nx, ny;
    std::vector<double> cl, cr, cb, ct;
};

double side_coef(const efsi_bc_side& s, int k) {
    if (s.type == EFSI_BC_DIRICHLET) return 2.0;
    if (s.type == EFSI_BC_MIXED && s.mask) return s.mask[k] ? 2.0 : 0.0;
    return 0.0;
}

void host_level_apply(const HostLevel& L, double ax, double ay, bool px, bool py, const std::vector<double>& x,
                      std::vector<double>& y) {
    const int nx = L.nx, ny = L.ny;
    y.assign((size_t)nx * ny, 0.0);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            size_t k = (size_t)i + (size_t)j * nx;
            double c = x[k], d = 0.0, off = 0.0;
            if (i > 0) { d += ax; off += ax * x[k - 1]; } else if (px) { d += ax; off += ax * x[k + nx - 1]; } else d += ax * L.cl[j];
            if (i < nx - 1) { d += ax; off += ax * x[k + 1]; } else if (px) { d += ax; off += ax * x[k - (nx - 1)]; } else d += ax * L.cr[j];
            if (j > 0) { d += ay; off += ay * x[k - nx]; } else if (py) { d += ay; off += ay * x[k + (size_t)(ny - 1) * nx]; } else d += ay * L.cb[i];
            if (j < ny - 1) { d += ay; off += ay * x[k + nx]; } else if (py) { d += ay; off += ay * x[k - (size_t)(ny - 1) * nx]; } else d += ay * L.ct[i];
            y[k] = d * c - off;
        }
}

// Inverse of the SPD (shifted if singular) coarse operator via Cholesky.
std::vector<double> coarse_inverse(const HostLevel& L, double ax, double ay, bool px, bool py, bool singular) {
    const int n = L.nx * L.ny;
    std::vector<double> A((size_t)n * n, 0.0), e(n, 0.0), col;
    for (int k = 0; k < n; ++k) {
        e[k] = 1.0;
        host_level_apply(L, ax, ay, px, py, e, col);
        for (int r = 0; r < n; ++r) A[(size_t)r * n + k] = col[r];
        e[k] = 0.0;
    }
    if (singular) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += A[(size_t)k * n + k];
        s /= (double)n * n;
        for (double& a : A) a += s;
    }
    // lower Cholesky, row-major, in place
    for (int j = 0; j < n; ++j) {
        double* Aj = &A[(size_t)j * n];
        double d = Aj[j];
        for (int k = 0; k < j; ++k) d -= Aj[k] * Aj[k];
        if (!(d > 0.0)) throw Err{EFSI_SOLVE, "coarse projection operator is not positive definite"};
        d = std::sqrt(d);
        Aj[j] = d;
        for (int i = j + 1; i < n; ++i) {
            double* Ai = &A[(size_t)i * n];
            double v = Ai[j];
            for (int k = 0; k < j; ++k) v -= Ai[k] * Aj[k];
            Ai[j] = v / d;
        }
    }
    // inverse of L (lower), then A^-1 = L^-T L^-1
    std::vector<double> Li((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) {
        Li[(size_t)i * n + i] = 1.0 / A[(size_t)i * n + i];
        for (int j = 0; j < i; ++j) {
            double s = 0.0;
            for (int k = j; k < i; ++k) s += A[(size_t)i * n + k] * Li[(size_t)k * n + j];
            Li[(size_t)i * n + j] = -s / A[(size_t)i * n + i];
        }
    }
    std::vector<double> inv((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
            for (int k = i; k < n; ++k) s += Li[(size_t)k * n + i] * Li[(size_t)k * n + j];
            inv[(size_t)i * n + j] = s;
            inv[(size_t)j * n + i] = s;
        }
    return inv;
}

// The 1-D kind of one direction of level 0 (SPEC_*), or -1 when the boundary factors of
// a side are not uniform (a mixed side) or the size is not a power of two.
int spectral_kind(bool periodic, const std::vector<double>& lo, const std::vector<double>& hi, int n) {
    if (n < 2 || (n & (n - 1)) != 0) return -1;
    if (periodic) return SPEC_P;
    auto uniform = [](const std::vector<double>& c) {
        for (double v : c)
            if (v != c[0]) return false;
        return c[0] == 0.0 || c[0] == 2.0;
    };
    if (!uniform(lo) || !uniform(hi)) return -1;
    const bool dl = lo[0] == 2.0, dr = hi[0] == 2.0;
    return dl ? (dr ? SPEC_DD : SPEC_DN) : (dr ? SPEC_ND : SPEC_NN);
}

// Twiddles and eigenvalues of one direction (long double host trigonometry).
SpecDir spectral_dir(efsi_handle* h, int kind, int n) {
    SpecDir d{};
    d.n = n;
    d.kind = kind;
    d.L = (kind == SPEC_ND || kind == SPEC_DN) ? 2 * n : n;
    d.logL = 0;
    while ((1 << d.logL) < d.L) ++d.logL;
    d.logn = 0;
    while ((1 << d.logn) < n) ++d.logn;
    d.inv_n = 1.0 / n;
    d.inv_L = 1.0 / d.L;
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<double2> w(std::max(1, d.L / 2)), mk(d.L);
    for (int t = 0; t < d.L / 2; ++t) {
        const long double a = 2.0L * pi * t / d.L;
        w[t] = make_double2((double)cosl(a), (double)-sinl(a));
    }
    for (int k = 0; k < d.L; ++k) {
        const long double a = pi * k / (2.0L * d.L);
        mk[k] = make_double2((double)cosl(a), (double)-sinl(a));
    }
    std::vector<double> mu(n);
    for (int k = 0; k < n; ++k) {
        long double v;
        switch (kind) {
            case SPEC_NN: v = 2.0L - 2.0L * cosl(pi * k / n); break;
            case SPEC_DD: v = 2.0L + 2.0L * cosl(pi * k / n); break;
            case SPEC_ND: case SPEC_DN: v = 2.0L - 2.0L * cosl(pi * (2 * k + 1) / (2.0L * n)); break;
            default: v = 2.0L - 2.0L * cosl(2.0L * pi * k / n); break;
        }
        mu[k] = k == 0 && (kind == SPEC_NN || kind == SPEC_P) ? 0.0 : (double)v;
    }
    auto upload = [&](const auto& v) {
        using T = typename std::decay_t<decltype(v)>::value_type;
        T* p = h->dalloc<T>(v.size());
        check_cuda(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "spectral upload");
        return p;
    };
    d.w = upload(w);
    d.mk = upload(mk);
    d.mu = upload(mu);
    return d;
}

// Enable the direct projection solve when both directions allow it and the per-block
// shared memory (FFT buffer + a tile of rows) fits.
void setup_spectral(efsi_handle* h, const HostLevel& L0, bool px, bool py) {
    Spectral& sp = h->pj.sp;
    sp = Spectral{};
    const int kx = spectral_kind(px, L0.cl, L0.cr, L0.nx), ky = spectral_kind(py, L0.cb, L0.ct, L0.ny);
    if (kx < 0 || ky < 0) return;
    const int Lx = (kx == SPEC_ND || kx == SPEC_DN) ? 2 * L0.nx : L0.nx;
    const int Ly = (ky == SPEC_ND || ky == SPEC_DN) ? 2 * L0.ny : L0.ny;
    // per block: L/2 twiddles, R padded FFT rows and (A, B) an R x (n + 8) tile of modes; at
    // most four rows, and at most ~112 KB so that two blocks share an SM
    constexpr size_t kBudget = 112 * 1024, kMax = 220 * 1024;
    auto smem = [](int L, int n, int R, bool tile) {
        return 16 * (size_t)(L / 2) + 16 * (size_t)R * spectral_row(L) + (tile ? 8 * (size_t)R * (n + 8) : 0);
    };
    auto rows = [&](int L, int n, bool tile) {  // a power of two dividing the row count
        int R = 4;
        while (R > 1 && smem(L, n, R, tile) > kBudget) R >>= 1;
        return smem(L, n, R, tile) <= kMax ? R : 0;
    };
    sp.rows_a = std::min(rows(Lx, L0.nx, true), L0.ny);
    sp.rows_b = std::min(rows(Ly, L0.ny, true), L0.nx);
    sp.rows_c = std::min(rows(Lx, L0.nx, false), L0.ny);
    if (sp.rows_a < 1 || sp.rows_b < 1 || sp.rows_c < 1) return;
    auto lg = [](int R) { int l = 0; while ((1 << l) < R) ++l; return l; };
    sp.lg_a = lg(sp.rows_a);
    sp.lg_b = lg(sp.rows_b);
    sp.lg_c = lg(sp.rows_c);
    sp.smem_a = smem(Lx, L0.nx, sp.rows_a, true);
    sp.smem_b = smem(Ly, L0.ny, sp.rows_b, true);
    sp.smem_c = smem(Lx, L0.nx, sp.rows_c, false);
    sp.dx = spectral_dir(h, kx, L0.nx);
    sp.dy = spectral_dir(h, ky, L0.ny);
    sp.on = true;
    check_cuda(spectral_configure(sp), "spectral kernel attributes");
}

void build_projection(efsi_handle* h, const efsi_config& cfg) {
    const int Nx = h->Nx, Ny = h->Ny;
    const bool px = cfg.mesh.periodic_x, py = cfg.mesh.periodic_y;
    const efsi_bc_setup& b = cfg.bc_correction;
    Projection& pj = h->pj;
    pj.nullspace = !(side_has_dirichlet(b.left) || side_has_dirichlet(b.right) || side_has_dirichlet(b.bottom) ||
                     side_has_dirichlet(b.top));
    std::vector<HostLevel> lv;
    HostLevel L0;
    L0.nx = Nx; L0.ny = Ny;
    L0.cl.resize(Ny); L0.cr.resize(Ny); L0.cb.resize(Nx); L0.ct.resize(Nx);
    for (int j = 0; j < Ny; ++j) { L0.cl[j] = px ? 0.0 : side_coef(b.left, j); L0.cr[j] = px ? 0.0 : side_coef(b.right, j); }
    for (int i = 0; i < Nx; ++i) { L0.cb[i] = py ? 0.0 : side_coef(b.bottom, i); L0.ct[i] = py ? 0.0 : side_coef(b.top, i); }
    lv.push_back(L0);
    while (true) {
        const HostLevel& F = lv.back();
        if ((long)F.nx * F.ny <= 1024 || (F.nx & 1) || (F.ny & 1) || F.nx < 4 || F.ny < 4) break;
        HostLevel C;
        C.nx = F.nx / 2; C.ny = F.ny / 2;
        C.cl.resize(C.ny); C.cr.resize(C.ny); C.cb.resize(C.nx); C.ct.resize(C.nx);
        for (int j = 0; j < C.ny; ++j) { C.cl[j] = 0.5 * (F.cl[2 * j] + F.cl[2 * j + 1]); C.cr[j] = 0.5 * (F.cr[2 * j] + F.cr[2 * j + 1]); }
        for (int i = 0; i < C.nx; ++i) { C.cb[i] = 0.5 * (F.cb[2 * i] + F.cb[2 * i + 1]); C.ct[i] = 0.5 * (F.ct[2 * i] + F.ct[2 * i + 1]); }
        lv.push_back(C);
        if (lv.size() >= 16) break;
    }
    if ((long)lv.back().nx * lv.back().ny > 1024)
        throw Err{EFSI_UNSUPPORTED, "the projection multigrid needs grid sizes that halve down to at most 1024 coarse cells"};
    const double ax = h->P.g.hy / h->P.g.hx, ay = h->P.g.hx / h->P.g.hy;
    pj.nlev = (int)lv.size();
    pj.nsm = h->P.nsm;
    pj.mixed = cfg.numerics.precision == EFSI_PRECISION_MIXED;
    for (int l = 0; l < pj.nlev; ++l) {
        MGLevel& M = pj.lev[l];
        const HostLevel& H = lv[l];
        M.nx = H.nx; M.ny = H.ny; M.ax = ax; M.ay = ay;
        auto up = [&](const std::vector<double>& v) {
            double* d = h->dalloc<double>(v.size());
            check_cuda(cudaMemcpy(d, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice), "mg upload");
            return d;
        };
        M.cl = up(H.cl); M.cr = up(H.cr); M.cb = up(H.cb); M.ct = up(H.ct);
        size_t n = (size_t)H.nx * H.ny;
        M.x = h->dalloc<double>(n); M.xo = h->dalloc<double>(n); M.b = h->dalloc<double>(n); M.r = h->dalloc<double>(n);
        if (pj.mixed) { M.xf = h->dalloc<float>(n); M.xof = h->dalloc<float>(n); M.bf = h->dalloc<float>(n); }
    }
    const HostLevel& C = lv.back();
    std::vector<double> inv = coarse_inverse(C, ax, ay, px, py, pj.nullspace);
    pj.nc = C.nx * C.ny;
    pj.coarse_inv = h->dalloc<double>(inv.size());
    check_cuda(cudaMemcpy(pj.coarse_inv, inv.data(), sizeof(double) * inv.size(), cudaMemcpyHostToDevice), "mg upload");
    if (pj.mixed) {
        std::vector<float> invf(inv.begin(), inv.end());
        pj.coarse_inv_f = h->dalloc<float>(invf.size());
        check_cuda(cudaMemcpy(pj.coarse_inv_f, invf.data(), sizeof(float) * invf.size(), cudaMemcpyHostToDevice),
                   "mg upload");
    }
    const size_t N = (size_t)Nx * Ny;
    pj.x = h->dalloc<double>(N); pj.r[0] = h->dalloc<double>(N); pj.r[1] = h->dalloc<double>(N); pj.z = pj.lev[0].xo;
    pj.p[0] = h->dalloc<double>(N); pj.p[1] = h->dalloc<double>(N);
    pj.Ap = h->dalloc<double>(N); pj.b = h->dalloc<double>(N); pj.rhs = h->dalloc<double>(N);
    pj.w = h->dalloc<double>(N); pj.s[0] = h->dalloc<double>(N); pj.s[1] = h->dalloc<double>(N);
    pj.Up = h->dalloc<double>(h->nu); pj.Vp = h->dalloc<double>(h->nv);
    if (cfg.numerics.projection_solver == EFSI_PROJECTION_AUTO) setup_spectral(h, L0, px, py);
}

// ---------------------------------------------------------------------------------------
// device status -> EFSI status
// ---------------------------------------------------------------------------------------
Err decode(const DevStatus& s) {
    char buf[512];
    static const char* fields[] = {"state.U", "state.V", "state.phi", "state.resource", "state.sigma_xx",
                                   "state.sigma_yy", "state.sigma_xy"};
    switch (s.code) {
        case DE_NONFINITE_STATE:
            snprintf(buf, sizeof buf, "%s contains non-finite values.", fields[std::min(std::max(s.where, 0), 6)]);
            return {EFSI_ARG, buf};
        case DE_STAGE1_CONSTRAINT:
            snprintf(buf, sizeof buf,
                     "The velocity entering stage 1 does not satisfy the prescribed divergence constraint. Maximum "
                     "|div(v)-G| = %.17g. Initialize the state with make_velocity_compatible! or provide a compatible velocity.",
                     s.value);
            return {EFSI_ARG, buf};
        case DE_INCOMPATIBLE:
            snprintf(buf, sizeof buf,
                     "The prescribed divergence constraint is incompatible with the Neumann/periodic correction "
                     "boundaries. The volume integral of the Poisson right-hand side is %.17g.",
                     s.value);
            return {EFSI_ARG, buf};
        case DE_PROJ_RESIDUAL:
            snprintf(buf, sizeof buf,
                     "Projection Poisson solve did not reach the required true-residual accuracy. Relative residual = %.17g, tolerance = 1e-08.",
                     s.value);
            return {EFSI_SOLVE, buf};
        case DE_PROJ_CONSTRAINT:
            snprintf(buf, sizeof buf, "Projection did not satisfy the prescribed divergence constraint. Weighted L2 residual = %.17g.", s.value);
            return {EFSI_SOLVE, buf};
        case DE_NON_SPD:
            snprintf(buf, sizeof buf,
                     "GeometricStructureExtension requires an SPD tensor; encountered a non-positive or non-finite eigenvalue (cell %d,%d).",
                     s.i + 1, s.j + 1);
            return {EFSI_DOMAIN, buf};
        case DE_NEUMANN_INFLOW:
            snprintf(buf, sizeof buf,
                     "A Neumann condition does not define the incoming advected state at face (%d,%d). Prescribe Dirichlet data for advective inflow.",
                     s.i + 1, s.j + 1);
            return {EFSI_ARG, buf};
        case DE_BAD_VISCOSITY: return {EFSI_ARG, "evaluated viscosity must be strictly positive everywhere."};
        case DE_BAD_DIFFUSIVITY: return {EFSI_ARG, "evaluated diffusivity must be strictly positive everywhere."};
        case DE_NONFINITE_SINK: return {EFSI_ARG, "Evaluated resource sink contains non-finite values."};
        case DE_LINEAR_NOCONV:  // _solve_linear_system! (TimeIntegrationIMEX.jl:637), stage numbered from 1
            snprintf(buf, sizeof buf, "%s stage %d GMRES residual is too large: %.17g",
                     s.where == 0 ? "velocity" : "resource", s.i + 1, s.value);
            return {EFSI_SOLVE, buf};
        default:
            snprintf(buf, sizeof buf, "device error %d", s.code);
            return {EFSI_ARG, buf};
    }
}

void fetch_dev(efsi_handle* h) {
    check_cuda(cudaMemcpyAsync(h->host, h->dev, sizeof(DevBlock), cudaMemcpyDeviceToHost, h->stream), "readback");
    check_cuda(cudaStreamSynchronize(h->stream), "step");
}

void raise_if_failed(efsi_handle* h) {
    if (h->host->st.code != 0) {
        Err e = decode(h->host->st);
        throw e;
    }
}

// ---------------------------------------------------------------------------------------
// per-call / per-step device bookkeeping
// ---------------------------------------------------------------------------------------
__global__ void k_reset_call(DevBlock* d) {  // status and batch counters
    d->st.code = 0;
    d->counter = 0;
    d->first_fail = -1;
    d->max_constraint = 0.0;
    d->max_trace = 0.0;
}
__global__ void k_begin_step(DevBlock* d, const double* __restrict__ times) {
    const int c = d->counter;
    d->t = times[2 * c];
    d->dt = times[2 * c + 1];
    d->max_constraint = 0.0;
    d->max_trace = 0.0;
    for (int k = 0; k < 12; ++k) (&d->iters[0][0])[k] = 0;
}
__global__ void k_end_step(DevBlock* d, StepRec* hist) {
    StepRec& r = hist[d->counter];
    r.v[0] = d->max_constraint;
    r.v[1] = d->max_trace;
    for (int k = 0; k < 5; ++k) r.v[2 + k] = d->report[k];
    r.nonspd = d->nonspd;
    for (int k = 0; k < 12; ++k) (&r.iters[0][0])[k] = (&d->iters[0][0])[k];
    if (d->st.code != 0 && d->first_fail < 0) d->first_fail = d->counter;
    d->counter += 1;
}

// ---------------------------------------------------------------------------------------
// CG solves: captured as a WHILE node, or driven from the host in predicted batches
// ---------------------------------------------------------------------------------------
enum { KIND_PROJ = 0, KIND_VISC = 1, KIND_DIFF = 2 };

template <class Init, class Body>
void solve(efsi_handle* h, int kind, int stage, CGScal* cg, int maxiter, int kernels_per_body, int iters_per_body,
           Init&& init, Body&& body) {
    int* iters_out = &h->dev->iters[kind][stage];
    if (h->capturing) {
        cudaGraph_t g;
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        check_cuda(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &g, &deps, &nd), "capture info");
        cudaGraphConditionalHandle ch;
        check_cuda(cudaGraphConditionalHandleCreate(&ch, g, 1, cudaGraphCondAssignDefault), "conditional handle");
        init(h->stream, iters_out, ch);
        check_cuda(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &g, &deps, &nd), "capture info");
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = ch;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        check_cuda(cudaGraphAddNode(&node, g, deps, nd, &np), "conditional node");
        check_cuda(cudaStreamUpdateCaptureDependencies(h->stream, &node, 1, cudaStreamSetCaptureDependencies),
                   "capture dependencies");
        cudaGraph_t bg = np.conditional.phGraph_out[0];
        check_cuda(cudaStreamBeginCaptureToGraph(h->stream2, bg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
                   "body capture");
        body(h->stream2, iters_out, ch);
        cudaGraph_t out;
        check_cuda(cudaStreamEndCapture(h->stream2, &out), "body capture");
        h->gs[h->recording ? 1 : 0].loops.push_back({kind, stage, kernels_per_body, iters_per_body});
        return;
    }
    init(h->stream, iters_out, (cudaGraphConditionalHandle)0);
    int bodies = 0;
    int batch = std::max(1, (h->pred[kind] + iters_per_body - 1) / iters_per_body);
    int* flags = h->done_pinned;  // iter, done, maxiter, conv (CGScal order)
    while (true) {
        for (int k = 0; k < batch && bodies * iters_per_body < maxiter; ++k, ++bodies)
            body(h->stream, iters_out, (cudaGraphConditionalHandle)0);
        h->launches += (long long)batch * kernels_per_body;
        check_cuda(cudaMemcpyAsync(flags, &cg->iter, 4 * sizeof(int), cudaMemcpyDeviceToHost, h->stream),
                   "cg readback");
        check_cuda(cudaStreamSynchronize(h->stream), "cg");
        if (flags[1] || bodies * iters_per_body >= maxiter) break;
        batch = 1;
    }
    h->pred[kind] = std::max(1, flags[0]);
}

// The Poisson solve K x = pj.b (MG-preconditioned CG) from the warm start q0.
void proj_solve(efsi_handle* h, int stage_slot, double reltol, const double* q0) {
    const Params& P = h->P;
    DevBlock* d = h->dev;
    const double N = (double)h->nc;
    if (h->pj.sp.on) {  // direct fast-diagonalisation solve inside a Richardson iteration
        solve(
            h, KIND_PROJ, stage_slot, &d->cg_proj, P.nu.projection_maxiter, 4, 1,
            [&](cudaStream_t s, int* io, cudaGraphConditionalHandle ch) {
                proj_spectral_init(P, h->pj, reltol, P.nu.projection_maxiter, q0, &d->cg_proj, &d->ps, h->slot[1],
                                   &d->st, io, ch, s);
                h->launches += 1;
            },
            [&](cudaStream_t s, int* io, cudaGraphConditionalHandle ch) {
                // x transform (2 x 8 N B), y pass (2 x 8 N), x pass + update (3 x 8 N),
                // residual (3 x 8 N)
                site(h, EFSI_SITE_SPECTRAL, 8.0 * N * 10.0,
                     [&] { proj_spectral_iter(P, h->pj, &d->cg_proj, &d->ps, h->slot[4], io, ch, s); });
            });
        return;
    }
    const double vb = proj_update_vcycle_bytes(h->pj);
    const int vk = proj_update_vcycle_kernels(h->pj);
    solve(
        h, KIND_PROJ, stage_slot, &d->cg_proj, P.nu.projection_maxiter,
        2 * (proj_matvec_kernels(h->pj) + vk), 2,
        [&](cudaStream_t s, int* io, cudaGraphConditionalHandle ch) {
            proj_cg_init(P, h->pj, reltol, P.nu.projection_maxiter, q0, &d->cg_proj, &d->ps, h->slot[1],
                         h->slot[2], &d->st, io, ch, s);
            h->launches += proj_init_kernels(h->pj);
        },
        [&](cudaStream_t s, int* io, cudaGraphConditionalHandle ch) {
            for (int par = 0; par < 2; ++par) {
                site(h, EFSI_SITE_PCG_MATVEC, 8.0 * N * 4.0,
                     [&] { proj_matvec(P, h->pj, par, &d->cg_proj, h->slot[3], s); });
                site(h, EFSI_SITE_VCYCLE, vb, [&] {
                    proj_update_vcycle(P, h->pj, par, &d->cg_proj, h->slot[4], h->slot[5], io, ch, s);
                });
            }
        });
}

// One projection of (compact predictor | full arrays) onto div = G, writing U_out/V_out/q.
void projection(efsi_handle* h, bool compact, const double* u_in, const double* v_in, const double* G, double* U_out,
                double* V_out, int stage_slot) {
    const Params& P = h->P;
    DevBlock* d = h->dev;
    const double N = (double)h->nc, nuv = (double)(h->nu + h->nv), g = G ? 1.0 : 0.0;
    site(h, EFSI_SITE_PROJ_RHS, 8.0 * (2.0 * nuv + N * (2.0 + g)),
         [&] { proj_rhs(P, h->pj, compact, u_in, v_in, G, &d->ps, h->slot[0], &d->st, h->stream); });
    proj_solve(h, stage_slot, P.nu.projection_reltol, h->q);
    site(h, EFSI_SITE_PROJ_FINISH, 8.0 * (4.0 * N + 2.0 * nuv + g * N), [&] {
        proj_finish(P, h->pj, G, h->q, U_out, V_out, &d->ps, &d->max_constraint, h->slot[6], h->slot[7], &d->st,
                    h->stream);
    });
    h->launches += 3;
}

void tendencies(efsi_handle* h, int s, const StageFields& f) {
    const Params& P = h->P;
    DevBlock* d = h->dev;
    const double N = (double)h->nc, nuv = (double)(h->nu + h->nv), g = f.G ? 1.0 : 0.0;
    const double* kappa = nullptr;
    if (P.md.capillarity == EFSI_CAP_DIFFUSE_AREA) {
        launch_capillary_curvature(P, f.phi, h->cap_a, h->cap_b, h->kappa, h->stream);
        kappa = h->kappa;
        h->launches += 1 + P.md.capillary_smoothing_passes;
    }
    // the supported body forces are steady, so the stage time does not enter the kernels
    site(h, EFSI_SITE_MOMENTUM, 8.0 * (nuv + N * (4.0 + g) + 2.0 * N),
         [&] { launch_momentum_rhs(P, 0.0, f, kappa, h->Eu[s], h->Ev[s], &d->st, h->stream); });
    if (P.md.phase_field_method == EFSI_PF_ACDI && P.md.pf_option) {
        launch_umax(P, f.U, f.V, &d->gamma_dyn, h->slot[0], h->stream);
        h->launches += 1;
    }
    site(h, EFSI_SITE_PHASE, 8.0 * (nuv + N * (2.0 + g)),
         [&] { launch_phase_rhs(P, f, &d->gamma_dyn, h->Ephi[s], &d->st, h->stream); });
    if (h->resource) launch_resource_rhs(P, f, h->Ec[s], h->diff ? h->Ic[s] : nullptr, &d->st, h->stream);
    site(h, EFSI_SITE_STRUCTURE, 8.0 * (nuv + N * (4.0 + g) + 3.0 * N),
         [&] { launch_structure_rhs(P, f, h->Exx[s], h->Eyy[s], h->Exy[s], &d->st, h->stream); });
    if (h->visc)
        site(h, EFSI_SITE_VISC_APPLY, 8.0 * N * (4.0 + (P.md.viscosity == EFSI_VISC_HARMONIC ? 1.0 : 0.0)),
             [&] { launch_viscous_apply(P, f.U, f.V, f.phi, h->Iu[s], h->Iv[s], h->stream); });
    h->launches += 3 + (h->resource ? 1 : 0) + (h->visc ? 1 : 0);
}

const double c_AI_diag[4] = {0.0, 4.0 / 15, 1.0 / 15, 1.0 / 6};

// Iterations a host-driven solve may enqueue: its limit plus the DIRECT continuation.
int solve_limit(const SolveOpts& o) { return o.maxiter + (o.fallback ? EFSI_LINEAR_HARD_CAP : 0); }

// The whole IMEX step (TimeIntegrationIMEX.jl:1159-1255) for the (t, dt) at the
// batch counter; identical for every step so that it can be captured once.
void enqueue_step(efsi_handle* h) {
    const Params& P = h->P;
    DevBlock* d = h->dev;
    cudaStream_t s = h->stream;
    const double* dtp = &d->dt;
    k_begin_step<<<1, 1, 0, s>>>(d, h->times_dev);
    if (h->recording) {  // tape slot of this step: the state it starts from
        adj_record(P, &d->counter, h->tape_stride(), 0, h->U, h->V, h->phi, h->sxx, h->syy, h->sxy, h->tape, s);
        h->launches += 1;
    }
    launch_prepare_step(P, h->U, h->V, h->phi, h->c, h->sxx, h->syy, h->sxy, h->sxn, h->syn, h->sxyn, &d->st, s);
    h->launches += 2;
    const double* Gp = h->growth ? h->G : nullptr;
    const double N = (double)h->nc;
    for (int st = 0; st < 4; ++st) {
        StageFields f;
        if (st == 0) {
            f = StageFields{h->U, h->V, h->phi, h->c, h->sxn, h->syn, h->sxyn, Gp};
        } else {
            bool rc = h->resource;
            const double nE = (st == 1) ? 1.0 : 2.0;
            site(h, EFSI_SITE_COMBINE, 8.0 * N * (4.0 + 4.0 * nE + 4.0 + (rc ? 2.0 + 2.0 * st : 0.0)), [&] {
                launch_combine_scalars(P, st, dtp, h->phi, h->sxn, h->syn, h->sxyn, h->c, h->Ephi, h->Exx, h->Eyy,
                                       h->Exy, rc ? h->Ec : nullptr, (rc && h->diff) ? h->Ic : nullptr, h->phis,
                                       h->sxs, h->sys, h->sxys, rc ? (h->diff ? h->rhs_c : h->cs) : nullptr, s);
            });
            h->launches += 1;
            const double* cstage = h->c;
            if (rc) {
                cstage = h->cs;
                if (h->diff) {
                    DtCoef alpha{dtp, c_AI_diag[st]};
                    const SolveOpts o = solve_opts(P.nu, P.nu.resource_method);
                    solve(
                        h, KIND_DIFF, st, &d->cg_diff, solve_limit(o), 6, 2,
                        [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
                            diff_init(P, alpha, o, h->c, h->rhs_c, h->phis, h->ds, &d->cg_diff, h->slot[0], io, ch,
                                      ss);
                            h->launches += 1;
                        },
                        [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
                            for (int k = 0; k < 2; ++k)
                                diff_iter(P, alpha, h->phis, h->ds, &d->cg_diff, h->slot[1], h->slot[2], io, ch, ss);
                        });
                    solve_status(&d->cg_diff, &d->st, 1, st, s);
                    h->launches += 1;
                }
            }
            f = StageFields{h->Us, h->Vs, h->phis, cstage, h->sxs, h->sys, h->sxys, Gp};
        }
        if (h->growth) {
            launch_growth(P, f.phi, f.c, h->G, &d->max_trace, h->slot[0], s);
            h->launches += 1;
        }
        if (st == 0) {
            launch_stage1_check(P, h->U, h->V, Gp, &d->max_constraint, h->slot[0], &d->st, s);
            h->launches += 1;
        } else {
            site(h, EFSI_SITE_VEL_RHS, 8.0 * N * (4.0 + 4.0 * st), [&] {
                launch_velocity_rhs(P, st, dtp, h->U, h->V, h->Eu, h->Ev, h->Iu, h->Iv, h->phis, h->rhs_u,
                                    h->rhs_v, s);
            });
            h->launches += 1;
            if (h->visc) {
                DtCoef alpha{dtp, c_AI_diag[st]};
                const SolveOpts o = solve_opts(P.nu, P.nu.velocity_method);
                const int maxit = solve_limit(o);
                if (h->mixed && visc_cheb_applies(P)) {
                    solve(
                        h, KIND_VISC, st, &d->cg_visc, maxit, 2, 2,
                        [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
                            site(h, EFSI_SITE_VISC_INIT, 8.0 * N * 10.0, [&] {
                                visc_cheb_init(P, alpha, o, h->U, h->V, h->rhs_u, h->rhs_v, h->vs, h->vm,
                                               &d->cg_visc, h->slot[0], io, ch, ss);
                            });
                            h->launches += 2;
                        },
                        [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
                            for (int k = 0; k < 2; ++k)  // FP32 e, r, d in and out: 48 B per point per launch
                                site(h, EFSI_SITE_VISC_CG, 4.0 * N * 12.0, [&] {
                                    visc_cheb_iter(P, alpha, h->rhs_u, h->rhs_v, h->vs, h->vm, k, &d->cg_visc,
                                                   h->slot[2], io, ch, ss);
                                });
                        });
                } else if (h->mixed) {
                    solve(
                        h, KIND_VISC, st, &d->cg_visc, maxit, 2, 2,
                        [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
                            site(h, EFSI_SITE_VISC_INIT, 8.0 * N * 10.0, [&] {
                                visc_mx_init(P, alpha, o, h->U, h->V, h->rhs_u, h->rhs_v, h->phis, h->vs, h->vm,
                                             &d->cg_visc, h->slot[0], io, ch, ss);
                            });
                            h->launches += 2;
                        },
                        [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
                            for (int k = 0; k < 2; ++k)  // FP32 vectors: 104 B per point per iteration
                                site(h, EFSI_SITE_VISC_CG, 8.0 * N * 13.0, [&] {
                                    visc_mx_iter(P, alpha, h->phis, h->rhs_u, h->rhs_v, h->vs, h->vm, k,
                                                 &d->cg_visc, h->slot[2], io, ch, ss);
                                });
                        });
                } else
                solve(
                    h, KIND_VISC, st, &d->cg_visc, maxit, 2, 2,
                    [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
                        site(h, EFSI_SITE_VISC_INIT, 8.0 * N * 18.0, [&] {
                            visc_init(P, alpha, o, h->U, h->V, h->rhs_u, h->rhs_v, h->phis, h->vs, &d->cg_visc,
                                      h->slot[0], h->slot[1], io, ch, ss);
                        });
                        h->launches += 3;
                    },
                    [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
                        for (int k = 0; k < 2; ++k)
                            site(h, EFSI_SITE_VISC_CG, 8.0 * N * 22.0, [&] {
                                visc_iter(P, alpha, h->phis, h->vs, k, &d->cg_visc, h->slot[2], io, ch, ss);
                            });
                    });
                solve_status(&d->cg_visc, &d->st, 0, st, s);
                h->launches += 1;
            } else {
                visc_enforce_dirichlet(P, h->rhs_u, h->rhs_v, h->vs.x_u, h->vs.x_v, s);
                h->launches += 1;
            }
            projection(h, true, h->vs.x_u, h->vs.x_v, Gp, h->Us, h->Vs, st);
        }
        if (st < 3) {
            if (h->recording && st > 0) {  // the stage fields the tendencies read
                adj_record(P, &d->counter, h->tape_stride(), st * h->block_words(), h->Us, h->Vs, h->phis, h->sxs,
                           h->sys, h->sxys, h->tape, s);
                h->launches += 1;
            }
            tendencies(h, st, f);
        }
    }
    site(h, EFSI_SITE_FINALIZE, 16.0 * (double)(h->nu + h->nv + 5 * h->nc), [&] {
        launch_finalize(P, h->Us, h->Vs, h->phis, h->resource ? h->cs : h->c, h->sxs, h->sys, h->sxys, h->U, h->V,
                        h->phi, h->c, h->sxx, h->syy, h->sxy, d->report, &d->nonspd, h->slot[0], h->slot[1], &d->st,
                        s);
    });
    if (h->recording) {  // phi of the committed state (the last stage's extension mask)
        adj_record(P, &d->counter, h->tape_stride(), 3 * h->block_words() - h->nu - h->nv, nullptr, nullptr, h->phi,
                   nullptr, nullptr, nullptr, h->tape, s);
        h->launches += 1;
    }
    k_end_step<<<1, 1, 0, s>>>(d, h->hist_dev);
    h->launches += 2;
}

// Capture the step once as a CUDA graph (CG loops become device-terminated WHILE
// nodes).  If the driver refuses any part, the handle falls back to host-driven
// stepping.
void ensure_graph(efsi_handle* h) {
    efsi_handle::GraphSlot& G = h->gs[h->recording ? 1 : 0];
    if (!h->use_graph || G.exec) return;
    h->capturing = true;
    G.loops.clear();
    h->launches = 0;
    bool ok = true;
    try {
        check_cuda(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "capture");
        try {
            enqueue_step(h);
        } catch (...) {
            cudaGraph_t junk = nullptr;
            cudaStreamCaptureStatus cs2 = cudaStreamCaptureStatusNone;
            if (cudaStreamIsCapturing(h->stream2, &cs2) == cudaSuccess && cs2 != cudaStreamCaptureStatusNone)
                cudaStreamEndCapture(h->stream2, &junk);  // a body graph is owned by its node
            junk = nullptr;
            cudaStreamEndCapture(h->stream, &junk);
            if (junk) cudaGraphDestroy(junk);
            throw;
        }
        cudaGraph_t g = nullptr;
        check_cuda(cudaStreamEndCapture(h->stream, &g), "capture");
        G.graph = g;
        check_cuda(cudaGraphInstantiate(&G.exec, g, 0), "graph instantiate");
    } catch (const Err&) {
        ok = false;
    }
    h->capturing = false;
    G.fixed_launches = h->launches;
    if (!ok) {
        cudaGetLastError();
        if (G.exec) { cudaGraphExecDestroy(G.exec); G.exec = nullptr; }
        if (G.graph) { cudaGraphDestroy(G.graph); G.graph = nullptr; }
        h->use_graph = false;
    }
}

// Kernel launches of the last graph step, from its recorded iteration counts.
long long graph_launches(const efsi_handle* h, const StepRec& r) {
    const efsi_handle::GraphSlot& G = h->gs[h->recording ? 1 : 0];
    long long n = G.fixed_launches;
    for (const auto& l : G.loops)  // a body runs whole; its later iterations return at once
        n += (long long)((r.iters[l.kind][l.stage] + l.iters_per_body - 1) / l.iters_per_body) * l.kernels_per_body;
    return n;
}

void fill_report_rec(const StepRec& r, efsi_step_report* out) {
    if (!out) return;
    out->maximum_projection_constraint_linf = r.v[0];
    out->maximum_growth_trace_error = r.v[1];
    out->minimum_phi = r.v[2];
    out->maximum_phi = r.v[3];
    out->minimum_resource = r.v[4];
    out->minimum_sigma_eigenvalue = r.v[5];
    out->maximum_abs_sigma_determinant_error = r.v[6];
    out->non_spd_cells = r.nonspd;
}

// n steps from (t0, dts): batches of up to kMaxBatch steps, each either graph
// launches or host-driven enqueues, with one host synchronisation per batch.
void run_steps(efsi_handle* h, double t0, const double* dts, int n, efsi_step_report* reports) {
    for (int k = 0; k < n; ++k)
        if (!std::isfinite(dts[k]) || !(dts[k] > 0)) throw Err{EFSI_ARG, "dt must be finite and strictly positive."};
    if (!std::isfinite(t0)) throw Err{EFSI_ARG, "t must be finite."};
    if (h->timed_site != EFSI_SITE_NONE) {
        // per-launch events cannot live inside graph loops: time sites host-driven
    } else {
        ensure_graph(h);
    }
    cudaGraphExec_t exec = h->gs[h->recording ? 1 : 0].exec;
    const bool graph = h->use_graph && exec && h->timed_site == EFSI_SITE_NONE;
    long long launches = 0;
    int32_t its[3][4] = {};
    k_reset_call<<<1, 1, 0, h->stream>>>(h->dev);
    double t = t0;
    for (int base = 0; base < n; base += kMaxBatch) {
        const int m = std::min(kMaxBatch, n - base);
        check_cuda(cudaStreamSynchronize(h->stream), "batch");  // the pinned time buffer is free again
        for (int k = 0; k < m; ++k) {
            h->times_pinned[2 * k] = t;
            h->times_pinned[2 * k + 1] = dts[base + k];
            t += dts[base + k];
        }
        check_cuda(cudaMemcpyAsync(h->times_dev, h->times_pinned, 2 * m * sizeof(double), cudaMemcpyHostToDevice,
                                   h->stream), "times");
        if (base > 0) {  // restart the batch counter, keep the sticky status
            check_cuda(cudaMemsetAsync(&h->dev->counter, 0, sizeof(int), h->stream), "counter");
        }
        for (int k = 0; k < m; ++k) {
            if (graph) {
                check_cuda(cudaGraphLaunch(exec, h->stream), "graph launch");
            } else {
                h->launches = 0;
                enqueue_step(h);
                launches += h->launches;
            }
        }
        check_cuda(cudaMemcpyAsync(h->hist_pinned, h->hist_dev, m * sizeof(StepRec), cudaMemcpyDeviceToHost, h->stream),
                   "history");
        fetch_dev(h);
        for (int k = 0; k < m; ++k) {
            const StepRec& r = h->hist_pinned[k];
            if (graph) launches += graph_launches(h, r);
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 4; ++b) its[a][b] += r.iters[a][b];
        }
        if (h->host->st.code != 0) {
            Err e = decode(h->host->st);
            int failed = base + std::max(h->host->first_fail, 0);
            if (n > 1) e.msg = "step " + std::to_string(failed + 1) + " of " + std::to_string(n) + ": " + e.msg;
            throw e;
        }
        if (reports)
            for (int k = 0; k < m; ++k) fill_report_rec(h->hist_pinned[k], &reports[base + k]);
    }
    h->stats.kernel_launches = launches;
    for (int b = 0; b < 4; ++b) {
        h->stats.projection_iterations[b] = its[KIND_PROJ][b];
        h->stats.velocity_iterations[b] = its[KIND_VISC][b];
        h->stats.resource_iterations[b] = its[KIND_DIFF][b];
    }
}

// ---------------------------------------------------------------------------------------
// differentiation form: sqrt(n) checkpoints, recomputed segments, reverse steps
// ---------------------------------------------------------------------------------------
constexpr double kAdjointReltol = 1e-13;  // the adjoint solves stand in for exact inverses

__global__ void k_set_dt(DevBlock* d, double dt) { d->dt = dt; }

void ensure_adjoint_buffers(efsi_handle* h) {
    if (h->adj) return;
    const size_t N = h->nc, nu = h->nu, nv = h->nv;
    const size_t nbx = (size_t)h->Nx + 1, nby = (size_t)h->Ny + 1;
    const size_t acc_words = 6 * N + 24 * N;
    const size_t words = 2 * (nu + nv + 4 * N) + acc_words + 2 * N + (nu + nv + N) + 3 * N + h->ckpt_stride() +
                         9 * N + 2 * nbx + 2 * nby + 1;
    double* p = nullptr;
    check_cuda(cudaMalloc(&p, words * sizeof(double)), "adjoint buffers");
    check_cuda(cudaMemset(p, 0, words * sizeof(double)), "adjoint buffers");
    h->adj = p;
    h->adj_words = words;
    efsi_handle::AdjBufs& a = h->ab;
    auto take = [&](size_t n) { double* q = p; p += n; return q; };
    a.lU = take(nu); a.lV = take(nv); a.lphi = take(N); a.lsxx = take(N); a.lsyy = take(N); a.lsxy = take(N);
    a.sU = take(nu); a.sV = take(nv); a.sphi = take(N); a.ssxx = take(N); a.ssyy = take(N); a.ssxy = take(N);
    a.acc = p;
    a.acc_words = acc_words;
    a.luu = take(N); a.luv = take(N); a.lphin = take(N); a.lsxn = take(N); a.lsyn = take(N); a.lscn = take(N);
    for (int q = 0; q < 3; ++q) {
        a.lEu[q] = take(N); a.lEv[q] = take(N); a.lIu[q] = take(N); a.lIv[q] = take(N);
        a.lEphi[q] = take(N); a.lExx[q] = take(N); a.lEyy[q] = take(N); a.lExy[q] = take(N);
    }
    a.lpu = take(N); a.lpv = take(N);
    a.zU = take(nu); a.zV = take(nv); a.zq = take(N);
    a.s0x = take(N); a.s0y = take(N); a.s0c = take(N);
    a.final_state = take(h->ckpt_stride());
    a.sc = AdjScratch{take(N), take(N), take(N), take(N), take(N), take(N), take(N), take(N), take(N)};
    a.bub = take(nbx); a.but = take(nbx); a.bvl = take(nby); a.bvr = take(nby); a.G = take(1);
}

// Copy the state and the warm start into (save) or out of (!save) a checkpoint slot.
void state_copy(efsi_handle* h, double* slot, bool save) {
    const size_t N = h->nc;
    double* f[8] = {h->U, h->V, h->phi, h->c, h->sxx, h->syy, h->sxy, h->q};
    const size_t n[8] = {h->nu, h->nv, N, N, N, N, N, N};
    size_t off = 0;
    for (int k = 0; k < 8; ++k) {
        double* dst = save ? slot + off : f[k];
        const double* src = save ? f[k] : slot + off;
        check_cuda(cudaMemcpyAsync(dst, src, n[k] * sizeof(double), cudaMemcpyDeviceToDevice, h->stream), "checkpoint");
        off += n[k];
    }
}

void zero(efsi_handle* h, double* p, size_t n) {
    check_cuda(cudaMemsetAsync(p, 0, n * sizeof(double), h->stream), "clear");
}

// Transposed projection of stage `st`: lam of the predictor (compact) from lam of the
// projected face velocities.
void adj_projection(efsi_handle* h, int st, const double* lU, const double* lV, double* lpu, double* lpv) {
    const Params& P = h->P;
    DevBlock* d = h->dev;
    adj_proj_rhs(P, h->pj, lU, lV, &d->ps, h->slot[0], h->stream);
    proj_solve(h, st, kAdjointReltol, h->ab.zq);
    proj_mean(P, h->pj, &d->ps, h->slot[6], h->stream);
    adj_proj_finish(P, h->pj, lU, lV, &d->ps, lpu, lpv, h->stream);
    h->launches += 3;
}

// Transposed viscous solve of stage `st` (the free block of I - dt a_ss A is symmetric):
// lam of the right-hand side in h->vs.x_u / x_v.
void adj_viscous(efsi_handle* h, int st, const double* phis, const double* ru, const double* rv) {
    const Params Ph = homogeneous(h->P);  // homogeneous Dirichlet rows: their data is not differentiated here
    DevBlock* d = h->dev;
    DtCoef alpha{&d->dt, c_AI_diag[st]};
    SolveOpts o{kAdjointReltol, EFSI_LINEAR_HARD_CAP, 0, h->P.nu.fallback_reltol};
    solve(
        h, KIND_VISC, st, &d->cg_visc, o.maxiter, 2, 2,
        [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
            visc_init(Ph, alpha, o, h->ab.zU, h->ab.zV, ru, rv, phis, h->vs, &d->cg_visc, h->slot[0], h->slot[1], io,
                      ch, ss);
            h->launches += 3;
        },
        [&](cudaStream_t ss, int* io, cudaGraphConditionalHandle ch) {
            for (int k = 0; k < 2; ++k) visc_iter(Ph, alpha, phis, h->vs, k, &d->cg_visc, h->slot[2], io, ch, ss);
        });
    solve_status(&d->cg_visc, &d->st, 0, st, h->stream);
    h->launches += 1;
}

// One step backwards (TimeIntegrationIMEX.jl:1159-1255 in reverse) from the tape slot of
// the step: ab.l* holds the adjoint of the state after the step on entry and the adjoint
// of the state before it on return; parameter adjoints accumulate.
void reverse_step(efsi_handle* h, int slot, double dt) {
    const Params& P = h->P;
    DevBlock* d = h->dev;
    cudaStream_t s = h->stream;
    efsi_handle::AdjBufs& a = h->ab;
    const size_t N = h->nc, nu = h->nu, nv = h->nv, B = h->block_words();
    const double* T = h->tape + (size_t)slot * h->tape_stride();
    auto fields = [&](const double* b) {
        return AdjIn{b, b + nu, b + nu + nv, b + nu + nv + N, b + nu + nv + 2 * N, b + nu + nv + 3 * N};
    };
    AdjIn f[3] = {fields(T), fields(T + B), fields(T + 2 * B)};
    const double* phi3 = T + 3 * B;
    k_set_dt<<<1, 1, 0, s>>>(d, dt);
    // stage 0 reads sigma_n' = the time-n extension reset of the recorded state
    adj_reset_sigma(P, f[0].phi, f[0].sxx, f[0].syy, f[0].sxy, a.s0x, a.s0y, a.s0c, s);
    f[0].sxx = a.s0x; f[0].syy = a.s0y; f[0].sxy = a.s0c;
    zero(h, a.acc, a.acc_words);
    const AdjOut so{a.sU, a.sV, a.sphi, a.ssxx, a.ssyy, a.ssxy};
    const AdjParam par{a.bub, a.but, a.bvl, a.bvr, a.G};
    auto tend = [&](int q) {
        return AdjTend{a.lEu[q], a.lEv[q], a.lIu[q], a.lIv[q], a.lEphi[q], a.lExx[q], a.lEyy[q], a.lExy[q]};
    };
    auto clear_stage = [&] {
        zero(h, a.sU, nu); zero(h, a.sV, nv);
        zero(h, a.sphi, N); zero(h, a.ssxx, N); zero(h, a.ssyy, N); zero(h, a.ssxy, N);
    };
    for (int st = 3; st >= 1; --st) {
        if (st == 3) {  // the last stage's fields are the state after the step
            const double* src[6] = {a.lU, a.lV, a.lphi, a.lsxx, a.lsyy, a.lsxy};
            double* dst[6] = {a.sU, a.sV, a.sphi, a.ssxx, a.ssyy, a.ssxy};
            const size_t n[6] = {nu, nv, N, N, N, N};
            for (int k = 0; k < 6; ++k)
                check_cuda(cudaMemcpyAsync(dst[k], src[k], n[k] * sizeof(double), cudaMemcpyDeviceToDevice, s),
                           "adjoint");
        } else {
            clear_stage();
            adj_tendencies(P, f[st], tend(st), so, par, a.sc, &d->st, s);
            h->launches += 12;
        }
        const double* phis = st == 3 ? phi3 : f[st].phi;
        // velocity path: projection, viscous solve, right-hand side
        adj_projection(h, st, a.sU, a.sV, a.lpu, a.lpv);
        const double* ru = a.lpu;
        const double* rv = a.lpv;
        if (h->visc) {
            adj_viscous(h, st, phis, a.lpu, a.lpv);
            ru = h->vs.x_u;
            rv = h->vs.x_v;
        }
        adj_velocity_rhs(P, st, dt, ru, rv, a.luu, a.luv, a.lEu, a.lEv, a.lIu, a.lIv, par, s);
        // scalar path: extension reset at phi_s, stage combination
        adj_combine(P, st, dt, phis, a.sphi, a.ssxx, a.ssyy, a.ssxy, a.lphin, a.lsxn, a.lsyn, a.lscn, a.lEphi,
                    a.lExx, a.lEyy, a.lExy, s);
        h->launches += 2;
    }
    clear_stage();
    adj_tendencies(P, f[0], tend(0), so, par, a.sc, &d->st, s);
    adj_step_start(P, f[0].phi, a.sU, a.sV, a.luu, a.luv, a.sphi, a.lphin, a.ssxx, a.ssyy, a.ssxy, a.lsxn, a.lsyn,
                   a.lscn, a.lU, a.lV, a.lphi, a.lsxx, a.lsyy, a.lsxy, s);
    h->launches += 15;
}

void require_adjoint(const efsi_handle* h) {
    const char* why = adjoint_unsupported(h->P, h->resource, h->growth);
    if (why[0]) throw Err{EFSI_UNSUPPORTED, why};
}

template <class F>
int guarded(efsi_handle* h, F&& f) {
    try {
        if (h) check_cuda(cudaSetDevice(h->device), "cudaSetDevice");
        f();
        return EFSI_OK;
    } catch (const Err& e) {
        if (h) h->err = e.msg; else g_create_error = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        if (h) h->err = e.what(); else g_create_error = e.what();
        return EFSI_CUDA;
    }
}

void h2d(efsi_handle* h, double* dst, const double* src, size_t n) {
    check_cuda(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, h->stream), "upload");
}
void d2h(efsi_handle* h, double* dst, const double* src, size_t n) {
    check_cuda(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "download");
}

}  // namespace

// =========================================================================================
// C entry points
// =========================================================================================
extern "C" {

int efsi_create(const efsi_config* cfg, efsi_handle** out) {
    if (out) *out = nullptr;
    auto h = std::make_unique<efsi_handle>();
    int st = guarded(nullptr, [&] {
        if (!cfg || !out) throw Err{EFSI_ARG, "config and output handle must not be NULL"};
        if (cfg->abi_version != EFSI_ABI_VERSION) throw Err{EFSI_ARG, "efsi_config ABI version mismatch"};
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Err{EFSI_CUDA, "no CUDA device is available"};
        check_cuda(cudaGetDevice(&h->device), "cudaGetDevice");
        const efsi_mesh& m = cfg->mesh;
        if (m.Nx < 2) throw Err{EFSI_ARG, "Nx must be at least 2."};
        if (m.Ny < 2) throw Err{EFSI_ARG, "Ny must be at least 2."};
        h->Nx = m.Nx; h->Ny = m.Ny;
        const double hx = m.Lx / m.Nx, hy = m.Ly / m.Ny;
        uniform_spacing(m.dx_c, m.Nx, hx, "dx_c");
        uniform_spacing(m.dy_c, m.Ny, hy, "dy_c");
        uniform_spacing(m.dx_f, m.Nx + 1, hx, "dx_f");
        uniform_spacing(m.dy_f, m.Ny + 1, hy, "dy_f");
        validate_models(*cfg);
        h->step_block = step_requirements(*cfg);
        check_cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
        check_cuda(cudaEventCreate(&h->call_ev[0]), "event");
        check_cuda(cudaEventCreate(&h->call_ev[1]), "event");
        Params& P = h->P;
        check_cuda(cudaDeviceGetAttribute(&P.nsm, cudaDevAttrMultiProcessorCount, h->device), "device attribute");
        check_cuda(solvers_configure(), "solver kernel attributes");
        P.g = GridD{m.Nx, m.Ny, m.periodic_x ? 1 : 0, m.periodic_y ? 1 : 0, hx, hy, 1.0 / hx, 1.0 / hy, m.Lx, m.Ly};
        const int Nx = m.Nx, Ny = m.Ny;
        upload_bcs(h.get(), cfg->bc_U, Ny, Nx + 1, P.bu, "U");
        upload_bcs(h.get(), cfg->bc_V, Ny + 1, Nx, P.bv, "V");
        upload_bcs(h.get(), cfg->bc_correction, Ny, Nx, P.bq, "correction");
        upload_bcs(h.get(), cfg->bc_phi, Ny, Nx, P.bphi, "phi");
        upload_bcs(h.get(), cfg->bc_resource, Ny, Nx, P.bc, "resource");
        upload_bcs(h.get(), cfg->bc_sigma_xx, Ny, Nx, P.bsxx, "sigma_xx");
        upload_bcs(h.get(), cfg->bc_sigma_yy, Ny, Nx, P.bsyy, "sigma_yy");
        upload_bcs(h.get(), cfg->bc_sigma_xy, Ny, Nx, P.bsxy, "sigma_xy");
        P.md = cfg->models;
        P.nu = cfg->numerics;
        if (P.md.growth_tensor == EFSI_GTENSOR_DIRECTIONAL) {  // normalised as in GrowthModels.jl:154-167
            double tx = P.md.growth_direction_x, ty = P.md.growth_direction_y, mag = std::hypot(tx, ty);
            if (!(mag > 0.0)) throw Err{EFSI_ARG, "Directional growth requires a non-zero direction vector."};
            P.md.growth_direction_x = tx / mag;
            P.md.growth_direction_y = ty / mag;
        }
        if (P.md.phase_field_method == EFSI_PF_ACDI) {
            const efsi_bc_side* ph[4] = {&cfg->bc_phi.left, &cfg->bc_phi.right, &cfg->bc_phi.bottom, &cfg->bc_phi.top};
            for (int k = 0; k < 4; ++k) {
                P.psi_bc[k] = 0.0;
                if (ph[k]->type == EFSI_BC_DIRICHLET && ph[k]->value) {
                    double p = std::min(std::max(ph[k]->value[0], 0.0), 1.0), e = P.md.pf_param[2];
                    P.psi_bc[k] = P.md.pf_param[1] * std::log((p + e) / (1.0 - p + e));
                }
            }
        }
        if (!(P.nu.projection_reltol > 0)) throw Err{EFSI_ARG, "projection_reltol must be positive."};
        if (!(P.nu.projection_maxiter > 0)) throw Err{EFSI_ARG, "projection_maxiter must be positive."};
        if (!(P.nu.linear_reltol > 0)) throw Err{EFSI_ARG, "Linear-solver reltol must be positive."};
        if (!(P.nu.linear_maxiter > 0)) throw Err{EFSI_ARG, "Linear-solver maxiter must be positive."};
        if (!(P.nu.fallback_reltol > 0)) throw Err{EFSI_ARG, "fallback_reltol must be positive."};
        for (int m : {P.nu.velocity_method, P.nu.resource_method})
            if (m != EFSI_LINEAR_DIRECT && m != EFSI_LINEAR_GMRES)
                throw Err{EFSI_ARG, "velocity_method must be :direct or :gmres."};
        h->visc = P.md.viscosity != EFSI_VISC_NONE;
        h->diff = P.md.diffusivity != EFSI_DIFF_NONE;
        h->growth = P.md.growth_source != EFSI_GROWTH_NONE;
        h->resource = !(P.md.growth_source == EFSI_GROWTH_NONE && P.md.diffusivity == EFSI_DIFF_NONE &&
                        P.md.resource_consumption == EFSI_CONSUMPTION_NONE);
        const size_t N = (size_t)Nx * Ny;
        h->nc = N; h->nu = (size_t)(Nx + 1) * Ny; h->nv = (size_t)Nx * (Ny + 1);
        h->U = h->dalloc<double>(h->nu); h->V = h->dalloc<double>(h->nv);
        h->phi = h->dalloc<double>(N); h->c = h->dalloc<double>(N);
        h->sxx = h->dalloc<double>(N); h->syy = h->dalloc<double>(N); h->sxy = h->dalloc<double>(N);
        h->q = h->dalloc<double>(N);
        h->Us = h->dalloc<double>(h->nu); h->Vs = h->dalloc<double>(h->nv);
        h->phis = h->dalloc<double>(N); h->cs = h->dalloc<double>(N);
        h->sxs = h->dalloc<double>(N); h->sys = h->dalloc<double>(N); h->sxys = h->dalloc<double>(N);
        h->sxn = h->dalloc<double>(N); h->syn = h->dalloc<double>(N); h->sxyn = h->dalloc<double>(N);
        h->G = h->dalloc<double>(N);
        for (int k = 0; k < 3; ++k) {
            h->Eu[k] = h->dalloc<double>(N); h->Ev[k] = h->dalloc<double>(N);
            h->Iu[k] = h->dalloc<double>(N); h->Iv[k] = h->dalloc<double>(N);
            h->Ephi[k] = h->dalloc<double>(N);
            h->Exx[k] = h->dalloc<double>(N); h->Eyy[k] = h->dalloc<double>(N); h->Exy[k] = h->dalloc<double>(N);
            h->Ec[k] = h->resource ? h->dalloc<double>(N) : nullptr;
            h->Ic[k] = (h->resource && h->diff) ? h->dalloc<double>(N) : nullptr;
        }
        h->rhs_u = h->dalloc<double>(N); h->rhs_v = h->dalloc<double>(N); h->rhs_c = h->dalloc<double>(N);
        if (P.md.capillarity == EFSI_CAP_DIFFUSE_AREA) {
            h->kappa = h->dalloc<double>(N); h->cap_a = h->dalloc<double>(N); h->cap_b = h->dalloc<double>(N);
        }
        ViscSolve& vs = h->vs;
        vs.x_u = h->dalloc<double>(N); vs.x_v = h->dalloc<double>(N);
        vs.p_u = h->dalloc<double>(N); vs.p_v = h->dalloc<double>(N);
        vs.dinv_u = h->dalloc<double>(N); vs.dinv_v = h->dalloc<double>(N);
        for (int k = 0; k < 2; ++k) {
            vs.r_u[k] = h->dalloc<double>(N); vs.r_v[k] = h->dalloc<double>(N);
            vs.w_u[k] = h->dalloc<double>(N); vs.w_v[k] = h->dalloc<double>(N);
            vs.s_u[k] = h->dalloc<double>(N); vs.s_v[k] = h->dalloc<double>(N);
        }
        h->mixed = P.nu.precision == EFSI_PRECISION_MIXED;
        if (P.nu.precision != EFSI_PRECISION_FP64 && !h->mixed) throw Err{EFSI_ARG, "unknown precision form"};
        if (h->mixed && h->visc) {
            ViscMixed& m = h->vm;
            for (int k = 0; k < 2; ++k) {
                m.r_u[k] = h->dalloc<float>(N); m.r_v[k] = h->dalloc<float>(N);
                m.w_u[k] = h->dalloc<float>(N); m.w_v[k] = h->dalloc<float>(N);
                m.s_u[k] = h->dalloc<float>(N); m.s_v[k] = h->dalloc<float>(N);
            }
            m.p_u = h->dalloc<float>(N); m.p_v = h->dalloc<float>(N);
            m.dinv_u = h->dalloc<float>(N); m.dinv_v = h->dalloc<float>(N);
            m.rR_u = h->dalloc<float>(N); m.rR_v = h->dalloc<float>(N);
            m.ring_w = h->dalloc<float>(visc_ring_cells(Nx, Ny) * kRingWeights);
        }
        ScalarSolve& ds = h->ds;
        ds.x = h->cs; ds.r = h->dalloc<double>(N);
        ds.p[0] = h->dalloc<double>(N); ds.p[1] = h->dalloc<double>(N); ds.Ap = h->dalloc<double>(N);
        ds.dinv = h->dalloc<double>(N);
        build_projection(h.get(), *cfg);
        // reduction slots sized for the largest launch grid ((Nx+1) x (Ny+1) points, 32x8 blocks)
        int maxBlocks = ((Nx + 1 + 31) / 32) * ((Ny + 1 + 7) / 8);
        for (RedSlot& r : h->slot) {
            r.part = h->dalloc<double>((size_t)maxBlocks * 6);
            r.ticket = h->dalloc<unsigned>(1);
            r.maxBlocks = maxBlocks;
        }
        h->dev = h->dalloc<DevBlock>(1);
        check_cuda(cudaMallocHost(&h->host, sizeof(DevBlock)), "pinned");
        check_cuda(cudaMallocHost(&h->done_pinned, 4 * sizeof(int)), "pinned");
        std::memset(h->host, 0, sizeof(DevBlock));
        for (RedSlot& r : h->dslot) {
            r.part = h->dalloc<double>((size_t)efsi_handle::kDiagBlocks * 32);
            r.ticket = h->dalloc<unsigned>(1);
            r.maxBlocks = efsi_handle::kDiagBlocks;
        }
        h->diag_dev = h->dalloc<double>(kDiagTotals);
        check_cuda(cudaMallocHost(&h->diag_pinned, kDiagTotals * sizeof(double)), "pinned");
        h->times_dev = h->dalloc<double>(2 * (size_t)kMaxBatch);
        h->hist_dev = h->dalloc<StepRec>(kMaxBatch);
        check_cuda(cudaMallocHost(&h->times_pinned, 2 * (size_t)kMaxBatch * sizeof(double)), "pinned");
        check_cuda(cudaMallocHost(&h->hist_pinned, (size_t)kMaxBatch * sizeof(StepRec)), "pinned");
        check_cuda(cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking), "stream");
        // default state: rest, sigma = I (the workspace's initial values)
        std::vector<double> ones(N, 1.0);
        check_cuda(cudaMemcpy(h->sxx, ones.data(), N * sizeof(double), cudaMemcpyHostToDevice), "init");
        check_cuda(cudaMemcpy(h->syy, ones.data(), N * sizeof(double), cudaMemcpyHostToDevice), "init");
        if (h->mixed && h->visc && visc_cheb_applies(P)) visc_ring_weights(P, h->vm.ring_w, h->stream);
        check_cuda(cudaDeviceSynchronize(), "create");
        *out = h.release();
    });
    return st;
}

void efsi_destroy(efsi_handle* h) { delete h; }

const char* efsi_last_error(const efsi_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int efsi_upload_state(efsi_handle* h, const double* U, const double* V, const double* phi, const double* c,
                      const double* sxx, const double* syy, const double* sxy) {
    return guarded(h, [&] {
        if (!U || !V || !phi || !sxx || !syy || !sxy) throw Err{EFSI_ARG, "state arrays must not be NULL"};
        h2d(h, h->U, U, h->nu); h2d(h, h->V, V, h->nv); h2d(h, h->phi, phi, h->nc);
        if (c) h2d(h, h->c, c, h->nc);
        else check_cuda(cudaMemsetAsync(h->c, 0, h->nc * sizeof(double), h->stream), "upload");
        h2d(h, h->sxx, sxx, h->nc); h2d(h, h->syy, syy, h->nc); h2d(h, h->sxy, sxy, h->nc);
        check_cuda(cudaStreamSynchronize(h->stream), "upload");
    });
}

int efsi_download_state(efsi_handle* h, double* U, double* V, double* phi, double* c, double* sxx, double* syy,
                        double* sxy) {
    return guarded(h, [&] {
        if (U) d2h(h, U, h->U, h->nu);
        if (V) d2h(h, V, h->V, h->nv);
        if (phi) d2h(h, phi, h->phi, h->nc);
        if (c) d2h(h, c, h->c, h->nc);
        if (sxx) d2h(h, sxx, h->sxx, h->nc);
        if (syy) d2h(h, syy, h->syy, h->nc);
        if (sxy) d2h(h, sxy, h->sxy, h->nc);
        check_cuda(cudaStreamSynchronize(h->stream), "download");
    });
}

int efsi_set_correction(efsi_handle* h, const double* q) {
    return guarded(h, [&] {
        if (q) h2d(h, h->q, q, h->nc);
        else check_cuda(cudaMemsetAsync(h->q, 0, h->nc * sizeof(double), h->stream), "correction");
        check_cuda(cudaStreamSynchronize(h->stream), "correction");
    });
}

int efsi_get_correction(efsi_handle* h, double* q) {
    return guarded(h, [&] {
        d2h(h, q, h->q, h->nc);
        check_cuda(cudaStreamSynchronize(h->stream), "correction");
    });
}

int efsi_make_velocity_compatible(efsi_handle* h, efsi_projection_result* r) {
    return guarded(h, [&] {
        const Params& P = h->P;
        DevBlock* d = h->dev;
        reset_call_stats(h);
        call_begin(h);
        k_reset_call<<<1, 1, 0, h->stream>>>(d);
        launch_prepare_step(P, h->U, h->V, h->phi, h->c, h->sxx, h->syy, h->sxy, h->sxn, h->syn, h->sxyn, &d->st,
                            h->stream);
        h->launches += 2;
        const double* Gp = nullptr;
        if (h->growth) {
            launch_growth(P, h->phi, h->c, h->G, &d->max_trace, h->slot[0], h->stream);
            Gp = h->G;
            h->launches += 1;
        }
        // project! of state.U/V in place: the predictor is copied to Up/Vp first.
        projection(h, false, h->U, h->V, Gp, h->U, h->V, 0);
        call_end(h);
        fetch_dev(h);
        raise_if_failed(h);
        if (r) {
            r->linear_relative_residual = h->host->ps.v[7];
            r->constraint_linf = h->host->ps.v[8];
            r->constraint_l2 = h->host->ps.v[9];
            r->compatibility_defect = h->pj.nullspace ? h->host->ps.v[0] : 0.0;
        }
        h->stats.projection_iterations[0] = h->host->iters[KIND_PROJ][0];
        h->stats.kernel_launches = h->launches;
    });
}

int efsi_integrate_step(efsi_handle* h, double t, double dt, efsi_step_report* report) {
    return guarded(h, [&] {
        if (!std::isfinite(t)) throw Err{EFSI_ARG, "t must be finite."};
        if (!std::isfinite(dt)) throw Err{EFSI_ARG, "dt must be finite."};
        if (!(dt > 0)) throw Err{EFSI_ARG, "dt must be strictly positive."};
        if (h->step_block.code != EFSI_OK) throw h->step_block;
        reset_call_stats(h);
        ensure_graph(h);
        call_begin(h);
        run_steps(h, t, &dt, 1, report);
        call_end(h);
    });
}

int efsi_integrate_step_host(efsi_handle* h, double* U, double* V, double* phi, double* c, double* sxx, double* syy,
                             double* sxy, double* q, double t, double dt, efsi_step_report* report) {
    return guarded(h, [&] {
        if (!U || !V || !phi || !sxx || !syy || !sxy) throw Err{EFSI_ARG, "state arrays must not be NULL"};
        if (!std::isfinite(t)) throw Err{EFSI_ARG, "t must be finite."};
        if (!std::isfinite(dt)) throw Err{EFSI_ARG, "dt must be finite."};
        if (!(dt > 0)) throw Err{EFSI_ARG, "dt must be strictly positive."};
        if (h->step_block.code != EFSI_OK) throw h->step_block;
        reset_call_stats(h);
        ensure_graph(h);
        call_begin(h);
        h2d(h, h->U, U, h->nu); h2d(h, h->V, V, h->nv); h2d(h, h->phi, phi, h->nc);
        if (c) h2d(h, h->c, c, h->nc);
        else check_cuda(cudaMemsetAsync(h->c, 0, h->nc * sizeof(double), h->stream), "upload");
        h2d(h, h->sxx, sxx, h->nc); h2d(h, h->syy, syy, h->nc); h2d(h, h->sxy, sxy, h->nc);
        if (q) h2d(h, h->q, q, h->nc);
        run_steps(h, t, &dt, 1, report);  // throws before any download when the step fails
        d2h(h, U, h->U, h->nu); d2h(h, V, h->V, h->nv); d2h(h, phi, h->phi, h->nc);
        if (c) d2h(h, c, h->c, h->nc);
        d2h(h, sxx, h->sxx, h->nc); d2h(h, syy, h->syy, h->nc); d2h(h, sxy, h->sxy, h->nc);
        if (q) d2h(h, q, h->q, h->nc);
        call_end(h);
    });
}

int efsi_step_n(efsi_handle* h, double t0, const double* dts, int32_t n, efsi_step_report* reports) {
    return guarded(h, [&] {
        if (n < 0 || (n > 0 && !dts)) throw Err{EFSI_ARG, "dts must hold n step sizes"};
        if (h->step_block.code != EFSI_OK) throw h->step_block;
        reset_call_stats(h);
        ensure_graph(h);
        call_begin(h);  // one event pair spans all n steps
        if (n > 0) run_steps(h, t0, dts, n, reports);
        call_end(h);
    });
}

int efsi_project(efsi_handle* h, double* U, double* V, const double* target, efsi_projection_result* r) {
    return guarded(h, [&] {
        DevBlock* d = h->dev;
        reset_call_stats(h);
        k_reset_call<<<1, 1, 0, h->stream>>>(d);
        h2d(h, h->Us, U, h->nu);
        h2d(h, h->Vs, V, h->nv);
        const double* Gp = nullptr;
        if (target) { h2d(h, h->G, target, h->nc); Gp = h->G; }
        projection(h, false, h->Us, h->Vs, Gp, h->Us, h->Vs, 0);
        fetch_dev(h);
        raise_if_failed(h);
        d2h(h, U, h->Us, h->nu);
        d2h(h, V, h->Vs, h->nv);
        check_cuda(cudaStreamSynchronize(h->stream), "project");
        if (r) {
            r->linear_relative_residual = h->host->ps.v[7];
            r->constraint_linf = h->host->ps.v[8];
            r->constraint_l2 = h->host->ps.v[9];
            r->compatibility_defect = h->pj.nullspace ? h->host->ps.v[0] : 0.0;
        }
        h->stats.projection_iterations[0] = h->host->iters[KIND_PROJ][0];
        h->stats.kernel_launches = h->launches;
    });
}

int efsi_phase_field_rhs(efsi_handle* h, const double* U, const double* V, const double* phi, const double* G,
                         double* rhs) {
    return guarded(h, [&] {
        DevBlock* d = h->dev;
        k_reset_call<<<1, 1, 0, h->stream>>>(d);
        h2d(h, h->Us, U, h->nu); h2d(h, h->Vs, V, h->nv); h2d(h, h->phis, phi, h->nc);
        const double* Gp = nullptr;
        if (G) { h2d(h, h->G, G, h->nc); Gp = h->G; }
        StageFields f{h->Us, h->Vs, h->phis, h->c, h->sxs, h->sys, h->sxys, Gp};
        if (h->P.md.phase_field_method == EFSI_PF_ACDI && h->P.md.pf_option)
            launch_umax(h->P, f.U, f.V, &d->gamma_dyn, h->slot[0], h->stream);
        launch_phase_rhs(h->P, f, &d->gamma_dyn, h->Ephi[0], &d->st, h->stream);
        fetch_dev(h);
        raise_if_failed(h);
        d2h(h, rhs, h->Ephi[0], h->nc);
        check_cuda(cudaStreamSynchronize(h->stream), "phase_field_rhs");
    });
}

int efsi_uwcdi_strang_step(efsi_handle* h, const double* U, const double* V, const double* phi, double dt,
                           int32_t x_first, double* out) {
    return guarded(h, [&] {
        if (h->P.md.phase_field_method != EFSI_PF_UWCDI) throw Err{EFSI_ARG, "context method is not UWCDI"};
        if (!U || !V || !phi || !out) throw Err{EFSI_ARG, "U, V, phi and out must not be NULL"};
        if (!std::isfinite(dt)) throw Err{EFSI_ARG, "dt must be finite."};
        DevBlock* d = h->dev;
        k_reset_call<<<1, 1, 0, h->stream>>>(d);
        h2d(h, h->Us, U, h->nu); h2d(h, h->Vs, V, h->nv); h2d(h, h->phis, phi, h->nc);
        // half sweep, full sweep in the other direction, half sweep (PhaseFieldMethods.jl:810-850)
        const int a1 = x_first ? 1 : 2, a2 = 3 - a1;
        const int axis[3] = {a1, a2, a1};
        const double step[3] = {0.5 * dt, dt, 0.5 * dt};
        const double* q = h->phis;
        for (int k = 0; k < 3; ++k) {
            if (step[k] == 0.0) continue;
            launch_strang_sweep(h->P, h->Us, h->Vs, q, h->Ephi[k], axis[k], step[k], &d->st, h->stream);
            q = h->Ephi[k];
        }
        fetch_dev(h);
        raise_if_failed(h);
        d2h(h, out, q, h->nc);
        check_cuda(cudaStreamSynchronize(h->stream), "uwcdi_strang_step");
    });
}

int efsi_structure_tensor_rhs(efsi_handle* h, const double* sxx, const double* syy, const double* sxy,
                              const double* U, const double* V, const double* phi, const double* G, double* rxx,
                              double* ryy, double* rxy) {
    return guarded(h, [&] {
        DevBlock* d = h->dev;
        k_reset_call<<<1, 1, 0, h->stream>>>(d);
        h2d(h, h->Us, U, h->nu); h2d(h, h->Vs, V, h->nv); h2d(h, h->phis, phi, h->nc);
        h2d(h, h->sxs, sxx, h->nc); h2d(h, h->sys, syy, h->nc); h2d(h, h->sxys, sxy, h->nc);
        const double* Gp = nullptr;
        if (G) { h2d(h, h->G, G, h->nc); Gp = h->G; }
        StageFields f{h->Us, h->Vs, h->phis, h->c, h->sxs, h->sys, h->sxys, Gp};
        launch_structure_rhs(h->P, f, h->Exx[0], h->Eyy[0], h->Exy[0], &d->st, h->stream);
        fetch_dev(h);
        raise_if_failed(h);
        d2h(h, rxx, h->Exx[0], h->nc); d2h(h, ryy, h->Eyy[0], h->nc); d2h(h, rxy, h->Exy[0], h->nc);
        check_cuda(cudaStreamSynchronize(h->stream), "structure_tensor_rhs");
    });
}

int efsi_momentum_explicit_rhs(efsi_handle* h, double t, const double* U, const double* V, const double* phi,
                               const double* sxx, const double* syy, const double* sxy, const double* G, double* Fx,
                               double* Fy) {
    return guarded(h, [&] {
        DevBlock* d = h->dev;
        k_reset_call<<<1, 1, 0, h->stream>>>(d);
        h2d(h, h->Us, U, h->nu); h2d(h, h->Vs, V, h->nv); h2d(h, h->phis, phi, h->nc);
        h2d(h, h->sxs, sxx, h->nc); h2d(h, h->sys, syy, h->nc); h2d(h, h->sxys, sxy, h->nc);
        const double* Gp = nullptr;
        if (G) { h2d(h, h->G, G, h->nc); Gp = h->G; }
        StageFields f{h->Us, h->Vs, h->phis, h->c, h->sxs, h->sys, h->sxys, Gp};
        const double* kappa = nullptr;
        if (h->P.md.capillarity == EFSI_CAP_DIFFUSE_AREA) {
            launch_capillary_curvature(h->P, f.phi, h->cap_a, h->cap_b, h->kappa, h->stream);
            kappa = h->kappa;
        }
        // full-face outputs land in the predictor buffers
        launch_momentum_full(h->P, t, f, kappa, h->pj.Up, h->pj.Vp, &d->st, h->stream);
        fetch_dev(h);
        raise_if_failed(h);
        d2h(h, Fx, h->pj.Up, h->nu); d2h(h, Fy, h->pj.Vp, h->nv);
        check_cuda(cudaStreamSynchronize(h->stream), "momentum_explicit_rhs");
    });
}

int efsi_apply_viscous_operator(efsi_handle* h, const double* phi, const double* uv, double* out) {
    return guarded(h, [&] {
        if (!h->visc) throw Err{EFSI_ARG, "viscosity model is inactive"};
        const int Nx = h->Nx, Ny = h->Ny;
        // build full MAC arrays whose compact part is uv (boundary faces unused)
        std::vector<double> Uf(h->nu, 0.0), Vf(h->nv, 0.0);
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                Uf[(size_t)i + (size_t)j * (Nx + 1)] = uv[(size_t)i + (size_t)j * Nx];
                Vf[(size_t)i + (size_t)j * Nx] = uv[h->nc + (size_t)i + (size_t)j * Nx];
            }
        h2d(h, h->Us, Uf.data(), h->nu); h2d(h, h->Vs, Vf.data(), h->nv); h2d(h, h->phis, phi, h->nc);
        launch_viscous_apply(h->P, h->Us, h->Vs, h->phis, h->Iu[0], h->Iv[0], h->stream);
        d2h(h, out, h->Iu[0], h->nc);
        d2h(h, out + h->nc, h->Iv[0], h->nc);
        check_cuda(cudaStreamSynchronize(h->stream), "apply_viscous_operator");
    });
}

int efsi_state_diagnostics(efsi_handle* h, const efsi_diag_config* cfg, efsi_diagnostics* out) {
    return guarded(h, [&] {
        if (!cfg || !out) throw Err{EFSI_ARG, "config and out must not be NULL"};
        if (cfg->nmax < 0 || cfg->nmax > EFSI_DIAG_MAX_MODES) throw Err{EFSI_ARG, "nmax must lie in 0..8"};
        launch_diagnostics(h->P, *cfg, h->U, h->V, h->phi, h->sxx, h->syy, h->sxy, h->dslot[0], h->dslot[1],
                           h->dslot[2], h->diag_dev, efsi_handle::kDiagBlocks, h->stream);
        check_cuda(cudaGetLastError(), "diagnostics");
        d2h(h, h->diag_pinned, h->diag_dev, kDiagTotals);
        check_cuda(cudaStreamSynchronize(h->stream), "diagnostics");
        const double* S = h->diag_pinned;
        const double* M = S + kDiagSums;
        const double* S2 = M + kDiagMaxes;
        const double eps = 2.220446049250313e-16, pi = 3.14159265358979323846, nan = std::nan("");
        const double mass = S[0];
        // phase_centroid (run_sugiyama_lid_driven_cavity.jl:497-498)
        if (!(mass > eps)) throw Err{EFSI_ARG, "Phase integral is too small to define a centroid."};
        efsi_diagnostics& o = *out;
        o = efsi_diagnostics{};
        o.x_centroid = S[1] / mass;
        o.y_centroid = S[2] / mass;
        o.phase_integral = mass;
        o.perimeter_proxy = S[3];
        o.mixed_layer_measure = S[4];
        // phase_geometry_diagnostics (:673-688)
        const double cxx = S2[0] / mass, cyy = S2[1] / mass, cxy = S2[2] / mass;
        const double gap = std::hypot(cxx - cyy, 2.0 * cxy);
        o.covariance_major = 0.5 * (cxx + cyy + gap);
        o.covariance_minor = 0.5 * (cxx + cyy - gap);
        o.aspect_ratio = o.covariance_minor > 0.0 ? std::sqrt(o.covariance_major / o.covariance_minor) : INFINITY;
        o.orientation_radians = gap > 100.0 * eps ? 0.5 * std::atan2(2.0 * cxy, cxx - cyy) : 0.0;
        o.R0 = S[3] / (2.0 * pi);
        o.effective_interface_width = S[3] > eps ? S[4] / S[3] : nan;
        o.effective_interface_cells = o.effective_interface_width / cfg->h_interface;
        for (int n = 0; n < cfg->nmax; ++n) {
            o.Rc[n] = S2[3 + n];
            o.Rs[n] = S2[3 + EFSI_DIAG_MAX_MODES + n];
            o.amplitudes[n] = std::hypot(o.Rc[n], o.Rs[n]);
        }
        // phase_bound_diagnostics (:709-722)
        o.phi_minimum = -M[0];
        o.phi_maximum = M[1];
        o.lower_violation = std::max(0.0, -o.phi_minimum);
        o.upper_violation = std::max(0.0, o.phi_maximum - 1.0);
        o.out_of_bounds_cells = (int64_t)S[8];
        // flow_diagnostics (:724-749) and the inputs of comparison_timestep_bounds
        o.maximum_speed = M[2];
        o.kinetic_energy = S[5];
        o.divergence_linf = M[3];
        o.divergence_l2 = std::sqrt(S[6] / S[7]);
        o.max_abs_U = M[4];
        o.max_abs_V = M[5];
        // tensor_region_diagnostics (:739-804)
        for (int r = 0; r < 4; ++r) {
            const double* s = S + 9 + 5 * r;
            const double* m = M + 6 + 6 * r;
            efsi_tensor_region& g = o.tensor[r];
            if (s[0] == 0.0 || s[1] == 0.0) {
                g = efsi_tensor_region{0, 0.0, nan, nan, nan, nan, nan, nan, 0, nan, nan};
            } else {
                g = efsi_tensor_region{(int64_t)s[0], s[1], -m[0], m[1], m[2], s[2] / s[1], -m[3], m[4],
                                       (int64_t)s[4], m[5], s[3] / s[1]};
            }
        }
    });
}

int efsi_forward_checkpointed(efsi_handle* h, double t0, const double* dts, int32_t n, int32_t every,
                              efsi_step_report* reports) {
    return guarded(h, [&] {
        if (n < 1 || !dts) throw Err{EFSI_ARG, "dts must hold n >= 1 step sizes"};
        if (h->step_block.code != EFSI_OK) throw h->step_block;
        require_adjoint(h);
        if (every <= 0) every = (int)std::ceil(std::sqrt((double)n));
        every = std::max(1, std::min(std::min(every, n), kMaxBatch));
        const int segs = (n + every - 1) / every;
        if (segs > h->adj_ckpt_cap) {
            if (h->ckpt) cudaFree(h->ckpt);
            h->ckpt = nullptr;
            h->adj_ckpt_cap = 0;
            check_cuda(cudaMalloc(&h->ckpt, (size_t)segs * h->ckpt_stride() * sizeof(double)), "checkpoints");
            h->adj_ckpt_cap = segs;
        }
        h->adj_n = 0;
        reset_call_stats(h);
        call_begin(h);
        long long launches = 0;
        int its[3][4] = {};
        double t = t0;
        for (int seg = 0; seg < segs; ++seg) {
            const int k0 = seg * every, m = std::min(every, n - k0);
            state_copy(h, h->ckpt + (size_t)seg * h->ckpt_stride(), true);
            run_steps(h, t, dts + k0, m, reports ? reports + k0 : nullptr);
            launches += h->stats.kernel_launches;
            for (int b = 0; b < 4; ++b) {
                its[0][b] += h->stats.projection_iterations[b];
                its[1][b] += h->stats.velocity_iterations[b];
                its[2][b] += h->stats.resource_iterations[b];
            }
            for (int k = 0; k < m; ++k) t += dts[k0 + k];
        }
        call_end(h);
        h->adj_n = n;
        h->adj_every = every;
        h->adj_t0 = t0;
        h->adj_dts.assign(dts, dts + n);
        h->stats.kernel_launches = launches;
        for (int b = 0; b < 4; ++b) {
            h->stats.projection_iterations[b] = its[0][b];
            h->stats.velocity_iterations[b] = its[1][b];
            h->stats.resource_iterations[b] = its[2][b];
        }
    });
}

int efsi_backward(efsi_handle* h, const double* lam_U, const double* lam_V, const double* lam_phi,
                  const double* lam_sxx, const double* lam_syy, const double* lam_sxy, double* grad_U,
                  double* grad_V, double* grad_phi, double* grad_sxx, double* grad_syy, double* grad_sxy,
                  efsi_gradient* grad) {
    return guarded(h, [&] {
        if (h->adj_n <= 0) throw Err{EFSI_ARG, "efsi_backward needs a preceding efsi_forward_checkpointed"};
        require_adjoint(h);
        ensure_adjoint_buffers(h);
        const int n = h->adj_n, every = h->adj_every, segs = (n + every - 1) / every;
        if (every > h->adj_tape_cap) {  // the recording graph holds the tape address: capture it again
            if (h->tape) cudaFree(h->tape);
            h->tape = nullptr;
            h->adj_tape_cap = 0;
            efsi_handle::GraphSlot& G = h->gs[1];
            if (G.exec) { cudaGraphExecDestroy(G.exec); G.exec = nullptr; }
            if (G.graph) { cudaGraphDestroy(G.graph); G.graph = nullptr; }
            check_cuda(cudaMalloc(&h->tape, (size_t)every * h->tape_stride() * sizeof(double)), "tape");
            h->adj_tape_cap = every;
        }
        efsi_handle::AdjBufs& a = h->ab;
        const size_t N = h->nc, nu = h->nu, nv = h->nv;
        const size_t nbx = (size_t)h->Nx + 1, nby = (size_t)h->Ny + 1;
        reset_call_stats(h);
        call_begin(h);
        state_copy(h, a.final_state, true);
        auto seed = [&](double* dst, const double* src, size_t m) {
            if (src) h2d(h, dst, src, m);
            else zero(h, dst, m);
        };
        seed(a.lU, lam_U, nu); seed(a.lV, lam_V, nv); seed(a.lphi, lam_phi, N);
        seed(a.lsxx, lam_sxx, N); seed(a.lsyy, lam_syy, N); seed(a.lsxy, lam_sxy, N);
        zero(h, a.bub, nbx); zero(h, a.but, nbx); zero(h, a.bvl, nby); zero(h, a.bvr, nby); zero(h, a.G, 1);
        std::vector<double> tseg(segs);
        double t = h->adj_t0;
        for (int seg = 0; seg < segs; ++seg) {
            tseg[seg] = t;
            for (int k = seg * every; k < std::min(n, (seg + 1) * every); ++k) t += h->adj_dts[k];
        }
        struct Recording {  // recording is on only while a segment is recomputed
            efsi_handle* h;
            ~Recording() { h->recording = false; }
        } guard{h};
        for (int seg = segs - 1; seg >= 0; --seg) {
            const int k0 = seg * every, m = std::min(every, n - k0);
            state_copy(h, h->ckpt + (size_t)seg * h->ckpt_stride(), false);
            h->recording = true;
            run_steps(h, tseg[seg], h->adj_dts.data() + k0, m, nullptr);  // recompute, recording the tape
            h->recording = false;
            for (int j = m - 1; j >= 0; --j) reverse_step(h, j, h->adj_dts[k0 + j]);
            fetch_dev(h);
            raise_if_failed(h);
        }
        state_copy(h, a.final_state, false);
        if (grad_U) d2h(h, grad_U, a.lU, nu);
        if (grad_V) d2h(h, grad_V, a.lV, nv);
        if (grad_phi) d2h(h, grad_phi, a.lphi, N);
        if (grad_sxx) d2h(h, grad_sxx, a.lsxx, N);
        if (grad_syy) d2h(h, grad_syy, a.lsyy, N);
        if (grad_sxy) d2h(h, grad_sxy, a.lsxy, N);
        if (grad) {
            d2h(h, &grad->elastic_coefficient, a.G, 1);
            if (grad->U_bottom) d2h(h, grad->U_bottom, a.bub, nbx);
            if (grad->U_top) d2h(h, grad->U_top, a.but, nbx);
            if (grad->V_left) d2h(h, grad->V_left, a.bvl, nby);
            if (grad->V_right) d2h(h, grad->V_right, a.bvr, nby);
        }
        call_end(h);
    });
}

int efsi_tendencies_adjoint(efsi_handle* h, const double* U, const double* V, const double* phi, const double* sxx,
                            const double* syy, const double* sxy, const double* lam_Eu, const double* lam_Ev,
                            const double* lam_Iu, const double* lam_Iv, const double* lam_Ephi,
                            const double* lam_Exx, const double* lam_Eyy, const double* lam_Exy, double* out_U,
                            double* out_V, double* out_phi, double* out_sxx, double* out_syy, double* out_sxy,
                            efsi_gradient* grad) {
    return guarded(h, [&] {
        if (!U || !V || !phi || !sxx || !syy || !sxy) throw Err{EFSI_ARG, "stage fields must not be NULL"};
        require_adjoint(h);
        ensure_adjoint_buffers(h);
        efsi_handle::AdjBufs& a = h->ab;
        const size_t N = h->nc, nu = h->nu, nv = h->nv;
        const size_t nbx = (size_t)h->Nx + 1, nby = (size_t)h->Ny + 1;
        DevBlock* d = h->dev;
        k_reset_call<<<1, 1, 0, h->stream>>>(d);
        h2d(h, h->Us, U, nu); h2d(h, h->Vs, V, nv); h2d(h, h->phis, phi, N);
        h2d(h, h->sxs, sxx, N); h2d(h, h->sys, syy, N); h2d(h, h->sxys, sxy, N);
        auto seed = [&](double* dst, const double* src, size_t m) {
            if (src) h2d(h, dst, src, m);
            else zero(h, dst, m);
        };
        seed(a.lEu[0], lam_Eu, N); seed(a.lEv[0], lam_Ev, N); seed(a.lIu[0], lam_Iu, N); seed(a.lIv[0], lam_Iv, N);
        seed(a.lEphi[0], lam_Ephi, N); seed(a.lExx[0], lam_Exx, N); seed(a.lEyy[0], lam_Eyy, N);
        seed(a.lExy[0], lam_Exy, N);
        zero(h, a.sU, nu); zero(h, a.sV, nv); zero(h, a.sphi, N);
        zero(h, a.ssxx, N); zero(h, a.ssyy, N); zero(h, a.ssxy, N);
        zero(h, a.bub, nbx); zero(h, a.but, nbx); zero(h, a.bvl, nby); zero(h, a.bvr, nby); zero(h, a.G, 1);
        adj_tendencies(h->P, AdjIn{h->Us, h->Vs, h->phis, h->sxs, h->sys, h->sxys},
                       AdjTend{a.lEu[0], a.lEv[0], a.lIu[0], a.lIv[0], a.lEphi[0], a.lExx[0], a.lEyy[0], a.lExy[0]},
                       AdjOut{a.sU, a.sV, a.sphi, a.ssxx, a.ssyy, a.ssxy},
                       AdjParam{a.bub, a.but, a.bvl, a.bvr, a.G}, a.sc, &d->st, h->stream);
        check_cuda(cudaGetLastError(), "tendencies adjoint");
        fetch_dev(h);
        raise_if_failed(h);
        if (out_U) d2h(h, out_U, a.sU, nu);
        if (out_V) d2h(h, out_V, a.sV, nv);
        if (out_phi) d2h(h, out_phi, a.sphi, N);
        if (out_sxx) d2h(h, out_sxx, a.ssxx, N);
        if (out_syy) d2h(h, out_syy, a.ssyy, N);
        if (out_sxy) d2h(h, out_sxy, a.ssxy, N);
        if (grad) {
            d2h(h, &grad->elastic_coefficient, a.G, 1);
            if (grad->U_bottom) d2h(h, grad->U_bottom, a.bub, nbx);
            if (grad->U_top) d2h(h, grad->U_top, a.but, nbx);
            if (grad->V_left) d2h(h, grad->V_left, a.bvl, nby);
            if (grad->V_right) d2h(h, grad->V_right, a.bvr, nby);
        }
        check_cuda(cudaStreamSynchronize(h->stream), "tendencies adjoint");
    });
}

int efsi_project_adjoint(efsi_handle* h, const double* lam_U, const double* lam_V, double* lam_U_in,
                         double* lam_V_in) {
    return guarded(h, [&] {
        if (!lam_U || !lam_V || !lam_U_in || !lam_V_in) throw Err{EFSI_ARG, "arrays must not be NULL"};
        ensure_adjoint_buffers(h);
        efsi_handle::AdjBufs& a = h->ab;
        DevBlock* d = h->dev;
        reset_call_stats(h);
        k_reset_call<<<1, 1, 0, h->stream>>>(d);
        h2d(h, a.sU, lam_U, h->nu);
        h2d(h, a.sV, lam_V, h->nv);
        adj_proj_rhs(h->P, h->pj, a.sU, a.sV, &d->ps, h->slot[0], h->stream);
        proj_solve(h, 0, kAdjointReltol, a.zq);
        proj_mean(h->P, h->pj, &d->ps, h->slot[6], h->stream);
        adj_proj_finish_full(h->P, h->pj, a.sU, a.sV, &d->ps, a.lU, a.lV, h->stream);
        fetch_dev(h);
        raise_if_failed(h);
        d2h(h, lam_U_in, a.lU, h->nu);
        d2h(h, lam_V_in, a.lV, h->nv);
        check_cuda(cudaStreamSynchronize(h->stream), "project adjoint");
        h->stats.projection_iterations[0] = h->host->iters[KIND_PROJ][0];
    });
}

int efsi_set_step_mode(efsi_handle* h, int32_t mode) {
    return guarded(h, [&] {
        if (mode != EFSI_STEP_GRAPH && mode != EFSI_STEP_HOST) throw Err{EFSI_ARG, "unknown step mode"};
        h->use_graph = mode == EFSI_STEP_GRAPH;
    });
}

int efsi_set_timed_site(efsi_handle* h, int32_t which) {
    return guarded(h, [&] {
        if (which < EFSI_SITE_NONE || which >= EFSI_SITE_COUNT) throw Err{EFSI_ARG, "unknown launch site"};
        h->timed_site = which;
        h->stats.site_launches = 0;
        h->stats.site_ms = 0.0;
        h->stats.site_bytes = 0.0;
        h->stats.step_bytes = 0.0;
        h->site_used = 0;
        h->site_bytes_pending = 0.0;
        h->step_bytes_pending = 0.0;
    });
}

}  // extern "C"

// =========================================================================================
// Allocation-free divergence residual (no counterpart in the reference)
// =========================================================================================
// Every other entry point works on a handle whose buffers efsi_create allocated.
// Some callers cannot allow a library to call cudaMalloc: hosts that hand all device
// memory out of their own pool allocator, and loops that must not meet the device-wide
// synchronisation that cudaMalloc/cudaFree may imply.  This entry point computes the
// stage-1 check of the IMEX step (max |div v - G|) on caller-owned device arrays with
// its reduction scratch in a fixed static device array instead of allocated buffers.
namespace {

constexpr int kNoAllocBlockX = 32, kNoAllocBlockY = 8;
// Block partials (two per block: max |div - G|, max |G|) and the completion ticket.
// 16384 blocks of 32x8 cells cover up to 4,194,304 cells (2048 x 2048); 256 KiB that
// every GPU which loads the library keeps until the process exits.
constexpr int kNoAllocMaxBlocks = 16384;
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxBlocks + 32];

// Device address of g_noalloc_scratch per device ordinal, looked up once per device.
std::mutex g_noalloc_mutex;
double* g_noalloc_base[256] = {};

double* noalloc_scratch(int device) {
    if (device < 0 || device >= 256) throw Err{EFSI_CUDA, "device ordinal out of range"};
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_base[device]) {
        double* p = nullptr;
        check_cuda(cudaGetSymbolAddress((void**)&p, g_noalloc_scratch), "scratch address");
        g_noalloc_base[device] = p;
    }
    return g_noalloc_base[device];
}

void require_device_pointer(const void* p, int device, const char* name) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        throw Err{EFSI_ARG, std::string(name) + " is not a CUDA device pointer"};
    }
    if (!((a.type == cudaMemoryTypeDevice && a.device == device) || a.type == cudaMemoryTypeManaged))
        throw Err{EFSI_ARG, std::string(name) + " must point to device (or managed) memory of the current device"};
}

// Same arithmetic as the stage-1 check of the step (k_stage1_check): per cell
// |(U(i+1)-U(i))/hx + (V(j+1)-V(j))/hy - G| and |G|, max-reduced over the grid.  The
// max reduction (fmax) would drop a NaN, so a non-finite cell value enters as +Inf:
// a velocity or target holding NaN or Inf can never report a finite residual.
__global__ void k_div_residual_noalloc(int Nx, int Ny, double ihx, double ihy, const double* __restrict__ U,
                                       const double* __restrict__ V, const double* __restrict__ G, double* out,
                                       RedSlot rs) {
    __shared__ double sh[64];
    const int i = blockIdx.x * kNoAllocBlockX + threadIdx.x, j = blockIdx.y * kNoAllocBlockY + threadIdx.y;
    double v[2] = {0.0, 0.0};
    if (i < Nx && j < Ny) {
        double div = (U[uidx(i + 1, j, Nx)] - U[uidx(i, j, Nx)]) * ihx + (V[vidx(i, j + 1, Nx)] - V[vidx(i, j, Nx)]) * ihy;
        double g = G ? G[cidx(i, j, Nx)] : 0.0;
        const double r = fabs(div - g), a = fabs(g);
        v[0] = isfinite(r) ? r : INFINITY;
        v[1] = isfinite(a) ? a : INFINITY;
    }
    double tot[2];
    if (grid_reduce<2, true>(v, rs, tot, sh) && threadIdx.x == 0 && threadIdx.y == 0) {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

}  // namespace

extern "C" {

int efsi_divergence_residual_noalloc(int32_t Nx, int32_t Ny, double Lx, double Ly, const double* U, const double* V,
                                     const double* G, double* out, void* stream) {
    return guarded(nullptr, [&] {
        if (Nx < 1 || Ny < 1) throw Err{EFSI_ARG, "Nx and Ny must be at least 1."};
        if (!(std::isfinite(Lx) && Lx > 0.0 && std::isfinite(Ly) && Ly > 0.0))
            throw Err{EFSI_ARG, "Lx and Ly must be finite and positive."};
        const long long bx = (Nx + kNoAllocBlockX - 1) / kNoAllocBlockX, by = (Ny + kNoAllocBlockY - 1) / kNoAllocBlockY;
        if (bx * by > kNoAllocMaxBlocks)
            throw Err{EFSI_ARG, "efsi_divergence_residual_noalloc: a " + std::to_string(Nx) + " x " + std::to_string(Ny) +
                                    " grid needs " + std::to_string(bx * by) + " reduction blocks of 32x8 cells; its "
                                    "fixed scratch holds at most " + std::to_string(kNoAllocMaxBlocks) +
                                    " (4,194,304 cells, e.g. 2048 x 2048)."};
        if (!U || !V || !out) throw Err{EFSI_ARG, "U, V and out must not be NULL."};
        int device = 0;
        check_cuda(cudaGetDevice(&device), "cudaGetDevice");
        require_device_pointer(U, device, "U");
        require_device_pointer(V, device, "V");
        if (G) require_device_pointer(G, device, "G");
        require_device_pointer(out, device, "out");
        double* base = noalloc_scratch(device);
        RedSlot rs;
        rs.part = base;
        rs.ticket = reinterpret_cast<unsigned*>(base + 2 * kNoAllocMaxBlocks);
        rs.maxBlocks = kNoAllocMaxBlocks;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // The ticket must start at zero; partials are written before they are read.
        check_cuda(cudaMemsetAsync(rs.ticket, 0, sizeof(unsigned), s), "scratch reset");
        const double hx = Lx / Nx, hy = Ly / Ny;
        k_div_residual_noalloc<<<dim3((unsigned)bx, (unsigned)by), dim3(kNoAllocBlockX, kNoAllocBlockY), 0, s>>>(
            Nx, Ny, 1.0 / hx, 1.0 / hy, U, V, G, out, rs);
        check_cuda(cudaGetLastError(), "launch");
    });
}

int efsi_get_stats(const efsi_handle* h, efsi_stats* s) {
    if (!h || !s) return EFSI_ARG;
    *s = h->stats;
    return EFSI_OK;
}

}  // extern "C"
