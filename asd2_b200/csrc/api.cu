// C-ABI entry points (include/asd2g.h): sessions, fields and the step
// operations, enqueued on the session's stream.
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <vector>

#include "asd2g.h"
#include "mg.cuh"
#include "ls32.cuh"

namespace asd2g {
// levelset.cu
void launch_center_vel(const Grid &g, const double *u, const double *v, double *tu, double *tv, cudaStream_t st);
void launch_ls_stage(int stage, const Grid &g, const double *phi_in, const double *tu, const double *tv,
                     const double *phi_n, double *out, const double *dt, cudaStream_t st);
void launch_reinit(const Grid &g, int mode, double max_atime, double *ls, double *ls0, double *w1, double *w2,
                   double *w3, cudaStream_t st);
void launch_absgrad(const Grid &g, bool sub, const double *ls, const double *ls0, double *out, cudaStream_t st);
void launch_sussman_only(const Grid &g, const double *ls, const double *ls0, const double *hd, double *out,
                         cudaStream_t st);
void launch_pointwise_ls(const Grid &g, int which, const double *a, double *out, cudaStream_t st);
void launch_weno_line(const double *F, double *FP, double *FM, double d, int n, cudaStream_t st);
void launch_weno_absgrad(const Grid &g, const double *ls, const double *ls0, double *out, cudaStream_t st);

DivH make_divh(double h) {
    DivH d;
    d.h = h;
    int e = 0;
    const double m = std::frexp(h, &e);
    d.pow2 = (m == 0.5) ? 1 : 0;
    d.inv = d.pow2 ? std::ldexp(1.0, 1 - e) : 1.0 / h;
    return d;
}

DivHT<float> make_divh_f(double h) {
    DivHT<float> d;
    d.h = (float)h;
    int e = 0;
    const float m = std::frexp(d.h, &e);
    d.pow2 = (m == 0.5f) ? 1 : 0;
    d.inv = d.pow2 ? std::ldexp(1.0f, 1 - e) : 1.0f / d.h;
    return d;
}

__global__ void k_set_scalar(double *p, double v) { *p = v; }
__global__ void k_fill(double *a, int64_t n, double v) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        a[k] = v;
}

// Statistics of a device-resident multi-step run (asd2g_run_steps).
struct RunStats {
    double max_res;      // largest final relative residual of the steps' solves
    long long iters;     // solver iterations summed over the steps
    int steps;           // steps executed
    int fail_step;       // first step whose solve failed or whose next dt is not positive and finite (-1: none)
    int fail_status;     // its solver status
    int loops;           // passes of the current solve's WHILE body
};

__global__ void k_run_reset(RunStats *rs) {
    rs->max_res = 0.0;
    rs->iters = 0;
    rs->steps = 0;
    rs->fail_step = -1;
    rs->fail_status = 0;
    rs->loops = 0;
}
// IF condition of the step: no earlier step failed.
__global__ void k_run_if(const RunStats *rs, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, rs->fail_step < 0 ? 1u : 0u);
}
// WHILE condition of the solve: not done; a hard cap on the passes ends the
// loop (status -7) whatever the solver state.
__global__ void k_run_while(KState *ks, RunStats *rs, int cap, cudaGraphConditionalHandle h) {
    const int loops = ++rs->loops;
    bool more = !ks->done;
    if (more && loops >= cap) {
        ks->status = -7;
        ks->done = 1;
        more = false;
    }
    cudaGraphSetConditional(h, more ? 1u : 0u);
}
// End of a step: accumulate, record a failure, hand the next dt to the next step.
__global__ void k_run_step_end(const KState *ks, RunStats *rs, double tol, double *dsc) {
    const bool conv = (ks->status == 0 && !(ks->res > tol)) || ks->status == 2;
    const double dtn = dsc[1];
    rs->iters += ks->it;
    rs->max_res = fmax(rs->max_res, ks->res);
    if ((!conv || !(dtn > 0.0) || !isfinite(dtn)) && rs->fail_step < 0) {
        rs->fail_step = rs->steps;
        rs->fail_status = conv ? -5 : ks->status;
    }
    rs->steps += 1;
    rs->loops = 0;
    dsc[0] = dtn;
}
void launch_run_reset(RunStats *rs, cudaStream_t st) { k_run_reset<<<1, 1, 0, st>>>(rs); }
void launch_run_if(const RunStats *rs, cudaGraphConditionalHandle h, cudaStream_t st) {
    k_run_if<<<1, 1, 0, st>>>(rs, h);
}
void launch_run_while(KState *ks, RunStats *rs, int cap, cudaGraphConditionalHandle h, cudaStream_t st) {
    k_run_while<<<1, 1, 0, st>>>(ks, rs, cap, h);
}
void launch_run_step_end(const KState *ks, RunStats *rs, double tol, double *dsc, cudaStream_t st) {
    k_run_step_end<<<1, 1, 0, st>>>(ks, rs, tol, dsc);
}
}  // namespace asd2g

using namespace asd2g;

namespace asd2g {
// The handler of every entry point's function-try-block: a C++ exception
// (a host allocation that failed, or any other) becomes a status code with
// its message in asd2g_last_error.  None crosses the C ABI.
int api_exception(const char *fn);
}  // namespace asd2g

namespace {
thread_local char g_err[512] = "";

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_check(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ASD2G_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return ASD2G_OK;
}

int kind_u(int side, int bc) {
    switch (bc) {
    case ASD2G_BC_PERIODIC: return K_PER;
    case ASD2G_BC_NEUMANN: return K_NEU;
    case ASD2G_BC_AXISYM: return side < 2 ? K_DIR : K_NEU;
    case ASD2G_BC_WALL: case ASD2G_BC_DIRICHLET: case ASD2G_BC_INLET: return K_DIR;
    case ASD2G_BC_OUTLET: return K_NEU;
    default: return K_NONE;
    }
}
int kind_v(int side, int bc) {
    switch (bc) {
    case ASD2G_BC_PERIODIC: return K_PER;
    case ASD2G_BC_NEUMANN: return K_NEU;
    case ASD2G_BC_AXISYM: return side < 2 ? K_NEU : K_DIR;
    case ASD2G_BC_WALL: case ASD2G_BC_DIRICHLET: case ASD2G_BC_INLET: return K_DIR;
    case ASD2G_BC_OUTLET: return K_NEU;
    default: return K_NONE;
    }
}
int kind_p(int bc) {
    switch (bc) {
    case ASD2G_BC_PERIODIC: return K_PER;
    case ASD2G_BC_NEUMANN: case ASD2G_BC_AXISYM: case ASD2G_BC_WALL: return K_NEU;
    case ASD2G_BC_DIRICHLET: case ASD2G_BC_INLET: case ASD2G_BC_OUTLET: case ASD2G_BC_PRESSURE: return K_DIR;
    case ASD2G_BC_LSFREE: return K_LSF;
    default: return K_NONE;
    }
}

// Validates p and derives the device-side grid and momentum constants of one
// session (or one batch instance).
int grid_from_params(const asd2g_params *p, Grid &g, MomConst &M) {
    if (p->nbc != NB) return fail(ASD2G_E_ARG, "num_bc_grid must be 3 (WENO5 needs three ghost layers), got %d", p->nbc);
    if (p->nx < 4 || p->ny < 4) return fail(ASD2G_E_ARG, "grid must be at least 4 x 4 cells, got %d x %d", p->nx, p->ny);
    if ((int64_t)(p->nx + 6) * (p->ny + 6) > (int64_t)1 << 31)
        return fail(ASD2G_E_ARG, "grid %d x %d too large", p->nx, p->ny);
    if (p->precision != ASD2G_PRECISION_FP64 && p->precision != ASD2G_PRECISION_MIXED)
        return fail(ASD2G_E_ARG, "precision %d: expected ASD2G_PRECISION_FP64 or _MIXED", p->precision);
    if (!(p->dx > 0.0) || !(p->dy > 0.0)) return fail(ASD2G_E_ARG, "dx, dy must be positive");
    for (int k = 0; k < 4; k++)
        if (p->bc_u[k] < 0 || p->bc_u[k] > 9 || p->bc_v[k] < 0 || p->bc_v[k] > 9 || p->bc_p[k] < 0 || p->bc_p[k] > 9)
            return fail(ASD2G_E_ARG, "boundary kind out of range");
    if (p->time_order < 0 || p->time_order > 2) return fail(ASD2G_E_ARG, "time_order must be 0, 1 or 2");
    g = Grid{};
    g.nx = p->nx;
    g.ny = p->ny;
    g.sx = p->nx + 2 * NB;
    g.sy = p->ny + 2 * NB;
    g.dx = p->dx;
    g.dy = p->dy;
    g.base_x = p->base_x;
    bool mirror = true, pinned = true;
    for (int k = 0; k < 4; k++) {
        g.ku[k] = kind_u(k, p->bc_u[k]);
        g.kv[k] = kind_v(k, p->bc_v[k]);
        g.kp[k] = kind_p(p->bc_p[k]);
        g.bp[k] = p->bc_p[k];
        g.bu[k] = p->bc_u[k];
        g.bv[k] = p->bc_v[k];
        g.cu[k] = p->bcc_u[k];
        g.cv[k] = p->bcc_v[k];
        g.cp[k] = p->bcc_p[k];
        mirror &= (g.kp[k] == K_NEU || g.kp[k] == K_DIR);
        pinned &= (p->bc_p[k] == ASD2G_BC_NEUMANN || p->bc_p[k] == ASD2G_BC_AXISYM || p->bc_p[k] == ASD2G_BC_WALL);
    }
    g.p_mirror = mirror ? 1 : 0;
    g.pinned = pinned ? 1 : 0;
    if (p->curvature != ASD2G_CURVATURE_REFERENCE && p->curvature != ASD2G_CURVATURE_DIVERGENCE)
        return fail(ASD2G_E_ARG, "curvature must be ASD2G_CURVATURE_REFERENCE or ASD2G_CURVATURE_DIVERGENCE");
    g.kappa_mode = p->curvature;
    if (p->precision == ASD2G_PRECISION_MIXED && !g.p_mirror)
        return fail(ASD2G_E_UNSUPPORTED, "mixed precision needs Neumann or Dirichlet pressure on all four sides");
    MomParams mp{p->rho_h, p->rho_l, p->mu_h, p->mu_l, p->sigma, p->gravity, p->cfl, p->g_axis, p->fix_gravity,
                 p->numbers_given, p->re, p->we, p->fr};
    M = make_momconst(g, mp);
    return ASD2G_OK;
}
}  // namespace

void asd2g::asd2g_set_error_text(const char *msg) { snprintf(g_err, sizeof(g_err), "%s", msg ? msg : ""); }

struct asd2g_session {
    asd2g_params prm;
    Grid g;
    MomConst M;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    size_t G = 0, N = 0;
    double *f[ASD2G_NFIELDS] = {};
    double *tu = nullptr, *tv = nullptr, *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
    double *ua = nullptr, *va = nullptr, *ub = nullptr, *vb = nullptr;
    Sys sys{};
    double *x = nullptr, *r = nullptr, *pa = nullptr, *pb = nullptr, *q = nullptr;
    double *rt = nullptr, *sv = nullptr, *t3 = nullptr;
    KState *ks = nullptr;
    KState *ks_host = nullptr;
    double *partial = nullptr;
    unsigned *counter = nullptr;
    double *dsc = nullptr;       // [0] dt of the step, [1] next dt, [2..3] residual sums, [4] counter
    double *dsc_host = nullptr;  // pinned mirror
    bool assembled = false;
    cudaGraphExec_t chunk_exec[6] = {};
    // learned preconditioner (ASD2G_SOLVER_UNET): network, features, output, scale
    asd2g_unet *pc_net = nullptr;
    float *pc_feats = nullptr, *pc_out = nullptr, *pc_scal = nullptr;
    FmDirs fm{};  // direction slots of the learned solver's truncated flexible CG
    int last_fallback = 0;
    int last_one_launch = 0;  // the last pressure solve ran as one kernel launch
    // multigrid preconditioner (allocated on first use)
    MgLevel lv[MG_MAX_LEVELS] = {};
    int nlev = 0;
    double *coarse_inv = nullptr, *z = nullptr;
    double *mg_partial = nullptr;  // per-tile partial sums of the V-cycle's fused dots
    unsigned *mgp_bar = nullptr;   // grid-barrier words of the one-launch solvers
    Ls32Work w32{};                // FP32 level-set work arrays (precision = mixed)
    double last_volume[2] = {0.0, 0.0};  // volume check of the last droplet step (sharp, smoothed)
    int64_t mg_partial_n = 0;
    int chunk_len = 64;
    // device-resident multi-step run (asd2g_run_steps): the step graph, the
    // streams its conditional bodies are captured on, its statistics
    cudaGraphExec_t run_exec = nullptr;
    // asd2g_ls_step replayed as one graph per reinitialisation mode (dt is
    // read from dsc[0] on the device, set before each replay)
    cudaGraphExec_t ls_exec[5] = {};
    // asd2g_droplet_step's phases before and after the solve, replayed as
    // graphs from the second call on (per reinitialisation mode / one)
    cudaGraphExec_t pre_exec[5] = {}, post_exec = nullptr;
    // asd2g_axi_step's phases likewise; the pre-solve graphs hold the level
    // set's boundary kinds of their capture (axi_ls_key) and are dropped
    // when a call brings others
    cudaGraphExec_t axi_pre_exec[5] = {}, axi_post_exec = nullptr;
    int axi_pre_calls[5] = {}, axi_post_calls = 0;
    int32_t axi_ls_key[4] = {-1, -1, -1, -1};
    double axi_ls_cst[4] = {0.0, 0.0, 0.0, 0.0};
    int pre_calls[5] = {}, post_calls = 0;
    int run_reinit = -1, run_maxit = -1;
    double run_tol = -1.0;
    cudaStream_t aux_st[2] = {};
    // staged copies: the session's copy stream and its events
    cudaStream_t copy_st = nullptr;
    cudaEvent_t ev_cmp = nullptr, ev_up = nullptr, ev_down = nullptr;
    RunStats *run_stats = nullptr, *run_stats_host = nullptr;
    std::vector<void *> allocs;
};

namespace {
int dalloc(asd2g_session *s, double **p, size_t n) {
    if (cudaMalloc(p, sizeof(double) * (n ? n : 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(ASD2G_E_NOMEM, "cudaMalloc of %zu doubles failed", n);
    }
    s->allocs.push_back(*p);
    return ASD2G_OK;
}

// V-cycle tile shape of a session (MG_SHAPES index): ASD2G_MG_TILE=0|1|2 in
// the environment, else the 16 x 32 tile, the fastest of the three for one
// system at 256^2 (922 / 830 / 828 solves/s) and 1024^2 (283 / 268 / 248).
static int mg_session_tile(int nx, int ny) {
    (void)nx;
    (void)ny;
    const char *forced = std::getenv("ASD2G_MG_TILE");
    if (forced && forced[0] >= '0' && forced[0] < '0' + MG_NSHAPES) return forced[0] - '0';
    return 0;
}

int mg_alloc(asd2g_session *s) {
    if (s->nlev) return ASD2G_OK;
    int dims[2 * MG_MAX_LEVELS];
    const int n = mg_levels_for(s->g.nx, s->g.ny, dims, MG_MAX_LEVELS);
    if (n < 2) return fail(ASD2G_E_UNSUPPORTED, "grid too small for the multigrid preconditioner");
    for (int l = 0; l < n; l++) {
        MgLevel &L = s->lv[l];
        L.nx = dims[2 * l];
        L.ny = dims[2 * l + 1];
        const size_t m = (size_t)L.nx * L.ny;
        float **arrs[] = {&L.diag, &L.ce, &L.cn, &L.f, &L.e, &L.ep};
        for (float **a : arrs) {
            if (cudaMalloc(a, sizeof(float) * m) != cudaSuccess) {
                cudaGetLastError();
                return fail(ASD2G_E_NOMEM, "multigrid level allocation failed");
            }
            s->allocs.push_back(*a);
            cudaMemsetAsync(*a, 0, sizeof(float) * m, s->st);
        }
    }
    int rc = dalloc(s, &s->coarse_inv, (size_t)MG_COARSE_CELLS * MG_COARSE_CELLS);
    if (rc == ASD2G_OK) rc = dalloc(s, &s->z, s->N);
    const int64_t np = mg_partial_len(s->g.nx, s->g.ny);
    if (rc == ASD2G_OK) rc = dalloc(s, &s->mg_partial, (size_t)np);
    if (rc) return rc;
    s->mg_partial_n = np;
    if (!mg_cta_prepare(s->lv, n)) return fail(ASD2G_E_UNSUPPORTED, "multigrid coarse cycle does not fit a CTA");
    mg_persist_prepare();  // process-wide kernel attribute, set before any capture can need it
    s->lv[0].tile = mg_session_tile(s->g.nx, s->g.ny);
    s->nlev = n;
    return ASD2G_OK;
}

int set_dt(asd2g_session *s, double dt) {
    k_set_scalar<<<1, 1, 0, s->st>>>(s->dsc, dt);
    return cuda_check("set dt");
}

bool valid_field(int f) { return f >= 0 && f < ASD2G_NFIELDS; }

int sync(asd2g_session *s) {
    const cudaError_t e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return fail(ASD2G_E_CUDA, "stream sync: %s", cudaGetErrorString(e));
    return ASD2G_OK;
}

bool stream_capturing(asd2g_session *s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s->st, &cs);
    return cs != cudaStreamCaptureStatusNone;
}

// false if a multigrid launch was refused (partial-sum buffer too small).
bool enqueue_iters(asd2g_session *s, int solver, int count) {
    const Grid &g = s->g;
    for (int k = 0; k < count; k++) {
        if (solver == ASD2G_SOLVER_MGPCG) {
            const double *po = k % 2 == 0 ? s->pa : s->pb;
            double *pn = k % 2 == 0 ? s->pb : s->pa;
            if (!launch_fcg_iter(s->sys, g.nx, g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, po, pn, s->q, s->z,
                                 s->ks, s->mg_partial, s->mg_partial_n, s->st))
                return false;
            // the FP64 residual check closes every run of 8 iterations
            if ((k % 8 == 7 || k == count - 1) &&
                !launch_fcg_check(s->sys, g.nx, g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, s->q, s->z, s->ks,
                                  s->mg_partial, s->mg_partial_n, s->st))
                return false;
        } else if (solver <= 1) {
            if (k % 2 == 0) launch_pcg_iter(g, s->sys, s->x, s->r, s->pa, s->pb, s->q, s->ks, s->partial, s->st);
            else launch_pcg_iter(g, s->sys, s->x, s->r, s->pb, s->pa, s->q, s->ks, s->partial, s->st);
        } else {
            launch_bicg_iter(g, s->sys, s->x, s->r, s->rt, s->pa, s->q, s->sv, s->t3, s->ks, s->partial, s->st);
        }
    }
    return true;
}
}  // namespace

extern "C" {

int asd2g_version(void) { return ASD2G_VERSION; }
const char *asd2g_last_error(void) { return g_err; }

int asd2g_create(const asd2g_params *p, void *stream, asd2g_session **out) try {
    if (!p || !out) return fail(ASD2G_E_ARG, "null argument");
    *out = nullptr;
    Grid g0{};
    MomConst M0{};
    int rc0 = grid_from_params(p, g0, M0);
    if (rc0) return rc0;
    asd2g_session *s = new (std::nothrow) asd2g_session();
    if (!s) return fail(ASD2G_E_NOMEM, "host allocation failed");
    s->prm = *p;
    s->g = g0;
    s->M = M0;
    Grid &g = s->g;
    s->G = (size_t)g.sx * g.sy;
    s->N = (size_t)g.nx * g.ny;
    if (stream) s->st = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
            delete s;
            return fail(ASD2G_E_CUDA, "cudaStreamCreate failed");
        }
        s->own_stream = true;
    }
    int rc = ASD2G_OK;
    const size_t G = s->G, N = s->N;
    for (int k = 0; k < ASD2G_NFIELDS && rc == ASD2G_OK; k++) rc = dalloc(s, &s->f[k], G);
    double **gw[] = {&s->tu, &s->tv, &s->w1, &s->w2, &s->w3, &s->ua, &s->va, &s->ub, &s->vb};
    for (double **pp : gw)
        if (rc == ASD2G_OK) rc = dalloc(s, pp, G);
    double **nw[] = {&s->sys.diag, &s->sys.cw, &s->sys.ce, &s->sys.cs, &s->sys.cn, &s->sys.minv, &s->sys.b,
                     &s->x, &s->r, &s->pa, &s->pb, &s->q, &s->rt, &s->sv};
    for (double **pp : nw)
        if (rc == ASD2G_OK) rc = dalloc(s, pp, N);
    if (rc == ASD2G_OK) rc = dalloc(s, &s->t3, 3 * N);
    if (rc == ASD2G_OK && p->precision == ASD2G_PRECISION_MIXED) {
        float **fw[LS32_ARRAYS] = {&s->w32.phi, &s->w32.ls0, &s->w32.a, &s->w32.b, &s->w32.tu, &s->w32.tv};
        for (float **pp : fw) {
            if (rc != ASD2G_OK) break;
            if (cudaMalloc(pp, sizeof(float) * G) != cudaSuccess) {
                cudaGetLastError();
                rc = fail(ASD2G_E_NOMEM, "FP32 work allocation failed");
            } else {
                s->allocs.push_back(*pp);
                cudaMemsetAsync(*pp, 0, sizeof(float) * G, s->st);
            }
        }
        // the Sussman band list: a 128-byte header holding the count, then nx * ny offsets
        const size_t nb = 32 + (size_t)p->nx * p->ny;
        void *bl = nullptr;
        if (rc == ASD2G_OK) {
            if (cudaMalloc(&bl, sizeof(int) * nb) != cudaSuccess) {
                cudaGetLastError();
                rc = fail(ASD2G_E_NOMEM, "FP32 band list allocation failed");
            } else {
                s->allocs.push_back(bl);
                cudaMemsetAsync(bl, 0, sizeof(int) * nb, s->st);
                s->w32.band_n = static_cast<unsigned *>(bl);
                s->w32.band = static_cast<int *>(bl) + 32;
            }
        }
    }
    if (rc == ASD2G_OK) rc = dalloc(s, &s->partial, 3 * RED_BLOCKS_MAX + 2 * DT_BLOCKS);
    if (rc == ASD2G_OK) rc = dalloc(s, &s->dsc, 8);
    if (rc == ASD2G_OK) {
        if (cudaMalloc(&s->ks, sizeof(KState)) != cudaSuccess) rc = fail(ASD2G_E_NOMEM, "KState allocation failed");
        else s->allocs.push_back(s->ks);
    }
    if (rc == ASD2G_OK) {
        if (cudaMalloc(&s->counter, sizeof(unsigned) * 4) != cudaSuccess) rc = fail(ASD2G_E_NOMEM, "counter allocation failed");
        else s->allocs.push_back(s->counter);
    }
    if (rc == ASD2G_OK) {  // grid-barrier words of the one-launch solvers
        if (cudaMalloc(&s->mgp_bar, 512 * sizeof(unsigned)) != cudaSuccess) rc = fail(ASD2G_E_NOMEM, "barrier words");
        else s->allocs.push_back(s->mgp_bar);
    }
    if (rc == ASD2G_OK && cudaMallocHost(&s->ks_host, sizeof(KState)) != cudaSuccess) rc = fail(ASD2G_E_NOMEM, "pinned alloc");
    if (rc == ASD2G_OK && cudaMallocHost(&s->dsc_host, sizeof(double) * 8) != cudaSuccess) rc = fail(ASD2G_E_NOMEM, "pinned alloc");
    if (rc != ASD2G_OK) {
        asd2g_destroy(s);
        return rc;
    }
    s->sys.pinned = g.pinned;
    // Fields and work arrays start at zero, like the reference's fresh vectors.
    for (void *a : s->allocs) (void)a;
    for (int k = 0; k < ASD2G_NFIELDS; k++) cudaMemsetAsync(s->f[k], 0, sizeof(double) * G, s->st);
    for (double **pp : gw) cudaMemsetAsync(*pp, 0, sizeof(double) * G, s->st);
    for (double **pp : nw) cudaMemsetAsync(*pp, 0, sizeof(double) * N, s->st);
    cudaMemsetAsync(s->t3, 0, sizeof(double) * 3 * N, s->st);
    cudaMemsetAsync(s->dsc, 0, sizeof(double) * 8, s->st);
    cudaMemsetAsync(s->counter, 0, sizeof(unsigned) * 4, s->st);
    cudaMemsetAsync(s->ks, 0, sizeof(KState), s->st);
    rc = sync(s);
    if (rc != ASD2G_OK) {
        asd2g_destroy(s);
        return rc;
    }
    *out = s;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_create");
}

int asd2g_destroy(asd2g_session *s) try {
    if (s && s->pc_net) asd2g_unet_set_stream(s->pc_net, nullptr);  // it must not keep this session's stream
    if (!s) return ASD2G_OK;
    if (s->st) cudaStreamSynchronize(s->st);
    for (auto &e : s->chunk_exec)
        if (e) cudaGraphExecDestroy(e);
    if (s->run_exec) cudaGraphExecDestroy(s->run_exec);
    for (auto &e : s->ls_exec)
        if (e) cudaGraphExecDestroy(e);
    for (auto &e : s->pre_exec)
        if (e) cudaGraphExecDestroy(e);
    if (s->post_exec) cudaGraphExecDestroy(s->post_exec);
    for (auto &e : s->axi_pre_exec)
        if (e) cudaGraphExecDestroy(e);
    if (s->axi_post_exec) cudaGraphExecDestroy(s->axi_post_exec);
    for (cudaStream_t a : s->aux_st)
        if (a) cudaStreamDestroy(a);
    if (s->copy_st) {
        cudaStreamSynchronize(s->copy_st);
        cudaStreamDestroy(s->copy_st);
    }
    for (cudaEvent_t e : {s->ev_cmp, s->ev_up, s->ev_down})
        if (e) cudaEventDestroy(e);
    if (s->run_stats_host) cudaFreeHost(s->run_stats_host);
    for (void *p : s->allocs) cudaFree(p);
    if (s->ks_host) cudaFreeHost(s->ks_host);
    if (s->dsc_host) cudaFreeHost(s->dsc_host);
    if (s->own_stream && s->st) cudaStreamDestroy(s->st);
    delete s;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_destroy");
}

int asd2g_sync(asd2g_session *s) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    return sync(s);
} catch (...) {
    return asd2g::api_exception("asd2g_sync");
}

int asd2g_field_ptr(asd2g_session *s, int field, double **dptr) try {
    if (!s || !dptr || !valid_field(field)) return fail(ASD2G_E_ARG, "bad field or null argument");
    *dptr = s->f[field];
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_field_ptr");
}

int asd2g_upload(asd2g_session *s, int field, const double *host) try {
    if (!s || !host || !valid_field(field)) return fail(ASD2G_E_ARG, "bad field or null argument");
    if (cudaMemcpyAsync(s->f[field], host, sizeof(double) * s->G, cudaMemcpyHostToDevice, s->st) != cudaSuccess)
        return cuda_check("upload");
    return sync(s);
} catch (...) {
    return asd2g::api_exception("asd2g_upload");
}

int asd2g_upload_async(asd2g_session *s, int field, const double *host) try {
    if (!s || !host || !valid_field(field)) return fail(ASD2G_E_ARG, "bad field or null argument");
    if (cudaMemcpyAsync(s->f[field], host, sizeof(double) * s->G, cudaMemcpyHostToDevice, s->st) != cudaSuccess)
        return cuda_check("upload");
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_upload_async");
}

// Staged copies: the session's copy stream waits for the compute work
// enqueued so far, copies, and records the upload or download event that
// asd2g_join_copies makes the compute stream wait for.
static int staged(asd2g_session *s, int field, void *host, bool up) {
    if (!s || !host || !valid_field(field)) return fail(ASD2G_E_ARG, "bad field or null argument");
    if (!s->copy_st) {
        if (cudaStreamCreateWithFlags(&s->copy_st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->ev_cmp, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->ev_up, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->ev_down, cudaEventDisableTiming) != cudaSuccess)
            return cuda_check("copy stream");
    }
    cudaEventRecord(s->ev_cmp, s->st);
    cudaStreamWaitEvent(s->copy_st, s->ev_cmp, 0);
    const size_t bytes = sizeof(double) * s->G;
    const cudaError_t e = up ? cudaMemcpyAsync(s->f[field], host, bytes, cudaMemcpyHostToDevice, s->copy_st)
                             : cudaMemcpyAsync(host, s->f[field], bytes, cudaMemcpyDeviceToHost, s->copy_st);
    if (e != cudaSuccess) return cuda_check(up ? "staged upload" : "staged download");
    cudaEventRecord(up ? s->ev_up : s->ev_down, s->copy_st);
    return cuda_check("staged copy");
}

int asd2g_upload_staged(asd2g_session *s, int field, const double *host) try {
    return staged(s, field, const_cast<double *>(host), true);
} catch (...) {
    return asd2g::api_exception("asd2g_upload_staged");
}

int asd2g_download_staged(asd2g_session *s, int field, double *host) { return staged(s, field, host, false); }

int asd2g_join_copies(asd2g_session *s, int which) try {
    if (!s || which < 1 || which > 3) return fail(ASD2G_E_ARG, "which: 1 uploads, 2 downloads, 3 both");
    if (!s->copy_st) return ASD2G_OK;
    if (which & 1) cudaStreamWaitEvent(s->st, s->ev_up, 0);
    if (which & 2) cudaStreamWaitEvent(s->st, s->ev_down, 0);
    return cuda_check("join copies");
} catch (...) {
    return asd2g::api_exception("asd2g_join_copies");
}

int asd2g_sync_copies(asd2g_session *s) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    if (s->copy_st && cudaStreamSynchronize(s->copy_st) != cudaSuccess) return cuda_check("copy stream");
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_sync_copies");
}

int asd2g_download(asd2g_session *s, int field, double *host) try {
    if (!s || !host || !valid_field(field)) return fail(ASD2G_E_ARG, "bad field or null argument");
    if (cudaMemcpyAsync(host, s->f[field], sizeof(double) * s->G, cudaMemcpyDeviceToHost, s->st) != cudaSuccess)
        return cuda_check("download");
    return sync(s);
} catch (...) {
    return asd2g::api_exception("asd2g_download");
}

int asd2g_copy_field(asd2g_session *s, int dst, int src) try {
    if (!s || !valid_field(dst) || !valid_field(src)) return fail(ASD2G_E_ARG, "bad field");
    if (dst == src) return ASD2G_OK;
    cudaMemcpyAsync(s->f[dst], s->f[src], sizeof(double) * s->G, cudaMemcpyDeviceToDevice, s->st);
    return cuda_check("copy_field");
} catch (...) {
    return asd2g::api_exception("asd2g_copy_field");
}

int asd2g_fill_field(asd2g_session *s, int field, double value) try {
    if (!s || !valid_field(field)) return fail(ASD2G_E_ARG, "bad field");
    k_fill<<<(int)((s->G + 255) / 256), 256, 0, s->st>>>(s->f[field], (int64_t)s->G, value);
    return cuda_check("fill_field");
} catch (...) {
    return asd2g::api_exception("asd2g_fill_field");
}

int asd2g_apply_bc_side(asd2g_session *s, int field, char kind, int side, int fill) try {
    if (!s || !valid_field(field) || side < 0 || side > 3) return fail(ASD2G_E_ARG, "bad field or side");
    int gk;
    if (kind == 'U' || kind == 'u') gk = 0;
    else if (kind == 'V' || kind == 'v') gk = 1;
    else if (kind == 'P' || kind == 'p') gk = 2;
    else return fail(ASD2G_E_ARG, "grid kind must be U, V or P");
    int k;
    if (fill == ASD2G_FILL_CONFIGURED) k = gk == 0 ? s->g.ku[side] : gk == 1 ? s->g.kv[side] : s->g.kp[side];
    else if (fill == ASD2G_FILL_PERIODIC) k = K_PER;
    else if (fill == ASD2G_FILL_NEUMANN) k = K_NEU;
    else if (fill == ASD2G_FILL_DIRICHLET) k = K_DIR;
    else if (fill == ASD2G_FILL_LSFREE && gk == 2) k = K_LSF;
    else return fail(ASD2G_E_ARG, "fill rule %d not defined for this grid", fill);
    launch_fill_side(s->g, s->f[field], gk, side, k, s->st);
    return cuda_check("apply_bc_side");
} catch (...) {
    return asd2g::api_exception("asd2g_apply_bc_side");
}

int asd2g_apply_bc(asd2g_session *s, int field, char kind) try {
    if (!s || !valid_field(field)) return fail(ASD2G_E_ARG, "bad field");
    if (kind == 'U' || kind == 'u') launch_fill_uv(s->g, s->f[field], nullptr, s->st);
    else if (kind == 'V' || kind == 'v') launch_fill_uv(s->g, nullptr, s->f[field], s->st);
    else if (kind == 'P' || kind == 'p') launch_fill_p(s->g, s->f[field], s->st);
    else return fail(ASD2G_E_ARG, "grid kind must be U, V or P");
    return cuda_check("apply_bc");
} catch (...) {
    return asd2g::api_exception("asd2g_apply_bc");
}

// ------------------------------------------------------------ level set --
// TVD-RK3 advection of LS with dt = dsc[0] (FP64 kernels).
static void enqueue_ls_advect(asd2g_session *s) {
    const Grid &g = s->g;
    double *ls = s->f[ASD2G_LS];
    launch_center_vel(g, s->f[ASD2G_U], s->f[ASD2G_V], s->tu, s->tv, s->st);
    launch_fill_p(g, ls, s->st);  // HJWENO5_LS_2D fills the input's ghosts first (levelset2d.cpp:99)
    launch_ls_stage(1, g, ls, s->tu, s->tv, ls, s->w1, s->dsc, s->st);
    launch_ls_stage(2, g, s->w1, s->tu, s->tv, ls, s->w2, s->dsc, s->st);
    launch_ls_stage(3, g, s->w2, s->tu, s->tv, ls, ls, s->dsc, s->st);
}

int asd2g_ls_advect(asd2g_session *s, double dt) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    int rc = set_dt(s, dt);
    if (rc) return rc;
    enqueue_ls_advect(s);
    return cuda_check("ls_advect");
} catch (...) {
    return asd2g::api_exception("asd2g_ls_advect");
}

int asd2g_ls_weno_rhs(asd2g_session *s, int ls, int uc, int vc, int out) try {
    if (!s || !valid_field(ls) || !valid_field(uc) || !valid_field(vc) || !valid_field(out))
        return fail(ASD2G_E_ARG, "bad field");
    if (out == ls || out == uc || out == vc) return fail(ASD2G_E_ARG, "out must differ from the inputs");
    launch_fill_p(s->g, s->f[ls], s->st);
    cudaMemsetAsync(s->f[out], 0, sizeof(double) * s->G, s->st);
    launch_ls_stage(0, s->g, s->f[ls], s->f[uc], s->f[vc], s->f[ls], s->f[out], s->dsc, s->st);
    return cuda_check("ls_weno_rhs");
} catch (...) {
    return asd2g::api_exception("asd2g_ls_weno_rhs");
}

int asd2g_reinit(asd2g_session *s, int mode) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    if (mode < 0 || mode > 4) return fail(ASD2G_E_ARG, "reinit mode %d out of range", mode);
    launch_reinit(s->g, mode, s->prm.ls_max_atime, s->f[ASD2G_LS], s->f[ASD2G_LS0], s->w1, s->w2, s->w3, s->st);
    return cuda_check("reinit");
} catch (...) {
    return asd2g::api_exception("asd2g_reinit");
}

int asd2g_subcell_eno(asd2g_session *s, int ls, int ls0, int out) try {
    if (!s || !valid_field(ls) || !valid_field(ls0) || !valid_field(out) || out == ls || out == ls0)
        return fail(ASD2G_E_ARG, "bad field");
    launch_absgrad(s->g, true, s->f[ls], s->f[ls0], s->f[out], s->st);
    return cuda_check("subcell_eno");
} catch (...) {
    return asd2g::api_exception("asd2g_subcell_eno");
}

int asd2g_eno(asd2g_session *s, int ls, int ls0, int out) try {
    if (!s || !valid_field(ls) || !valid_field(ls0) || !valid_field(out) || out == ls || out == ls0)
        return fail(ASD2G_E_ARG, "bad field");
    launch_absgrad(s->g, false, s->f[ls], s->f[ls0], s->f[out], s->st);
    return cuda_check("eno");
} catch (...) {
    return asd2g::api_exception("asd2g_eno");
}

int asd2g_sussman_constraint(asd2g_session *s, int ls, int ls0, int hd, int out) try {
    if (!s || !valid_field(ls) || !valid_field(ls0) || !valid_field(hd) || !valid_field(out) || out == ls ||
        out == ls0 || out == hd)
        return fail(ASD2G_E_ARG, "bad field");
    launch_sussman_only(s->g, s->f[ls], s->f[ls0], s->f[hd], s->f[out], s->st);
    return cuda_check("sussman_constraint");
} catch (...) {
    return asd2g::api_exception("asd2g_sussman_constraint");
}

int asd2g_heaviside_deriv(asd2g_session *s, int ls, int out) try {
    if (!s || !valid_field(ls) || !valid_field(out)) return fail(ASD2G_E_ARG, "bad field");
    launch_pointwise_ls(s->g, 0, s->f[ls], s->f[out], s->st);
    return cuda_check("heaviside_deriv");
} catch (...) {
    return asd2g::api_exception("asd2g_heaviside_deriv");
}

int asd2g_smoothed_sign(asd2g_session *s, int ls, int out) try {
    if (!s || !valid_field(ls) || !valid_field(out)) return fail(ASD2G_E_ARG, "bad field");
    launch_pointwise_ls(s->g, 1, s->f[ls], s->f[out], s->st);
    return cuda_check("smoothed_sign");
} catch (...) {
    return asd2g::api_exception("asd2g_smoothed_sign");
}

// Advection + reinitialisation of LS with dt = dsc[0]: the FP32 path for
// mixed sessions, else the FP64 kernels (asd2g_ls_advect + asd2g_reinit).
static void enqueue_ls_step(asd2g_session *s, int reinit_mode) {
    if (s->prm.precision == ASD2G_PRECISION_MIXED) {
        launch_fill_p(s->g, s->f[ASD2G_LS], s->st);
        launch_ls_step32(s->g, reinit_mode, s->prm.ls_max_atime, s->f[ASD2G_U], s->f[ASD2G_V], s->dsc,
                         s->f[ASD2G_LS], s->w32, s->st);
    } else {
        enqueue_ls_advect(s);
        launch_reinit(s->g, reinit_mode, s->prm.ls_max_atime, s->f[ASD2G_LS], s->f[ASD2G_LS0], s->w1, s->w2, s->w3,
                      s->st);
    }
}

// The step's launches (about 20 at the default reinitialisation) are
// captured once per mode and replayed as one graph: at small grids the
// kernels take a few microseconds each and launching them one by one from
// the host is what bounds the step.  Inside a caller's own stream capture
// they are enqueued directly.
int asd2g_ls_step(asd2g_session *s, double dt, int reinit_mode) try {
    NvtxRange nv("asd2g_ls_step");
    if (!s) return fail(ASD2G_E_ARG, "null session");
    if (reinit_mode < 0 || reinit_mode > 4) return fail(ASD2G_E_ARG, "reinit mode %d out of range", reinit_mode);
    if (s->prm.precision == ASD2G_PRECISION_MIXED && !ls32_supported(s->g, reinit_mode))
        return fail(ASD2G_E_UNSUPPORTED, "mixed precision implements reinit modes 0, 2 and 4, not %d", reinit_mode);
    int rc = set_dt(s, dt);
    if (rc) return rc;
    if (stream_capturing(s)) {
        enqueue_ls_step(s, reinit_mode);
        return cuda_check("ls_step");
    }
    if (!s->ls_exec[reinit_mode]) {
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();  // a stream that cannot be captured: launch one by one
            enqueue_ls_step(s, reinit_mode);
            return cuda_check("ls_step");
        }
        enqueue_ls_step(s, reinit_mode);
        if (cudaStreamEndCapture(s->st, &graph) != cudaSuccess) return cuda_check("ls_step capture end");
        cudaGraphExec_t ex = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&ex, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_check("ls_step graph instantiate");
        s->ls_exec[reinit_mode] = ex;
    }
    if (cudaGraphLaunch(s->ls_exec[reinit_mode], s->st) != cudaSuccess) return cuda_check("ls_step graph launch");
    return cuda_check("ls_step");
} catch (...) {
    return asd2g::api_exception("asd2g_ls_step");
}

int asd2g_last_volume(asd2g_session *s, double *sharp, double *smooth) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    if (sharp) *sharp = s->last_volume[0];
    if (smooth) *smooth = s->last_volume[1];
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_last_volume");
}

int asd2g_volume(asd2g_session *s, double *sharp, double *smooth) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    launch_heaviside(s->g, s->f[ASD2G_LS], s->f[ASD2G_H], s->f[ASD2G_HS], s->st);
    launch_volume(s->g, s->f[ASD2G_H], s->f[ASD2G_HS], s->partial, s->counter + 1, s->dsc + 5, s->st);
    cudaMemcpyAsync(s->dsc_host + 5, s->dsc + 5, sizeof(double) * 2, cudaMemcpyDeviceToHost, s->st);
    int rc = sync(s);
    if (rc) return rc;
    if (sharp) *sharp = s->dsc_host[5];
    if (smooth) *smooth = s->dsc_host[6];
    return cuda_check("volume");
} catch (...) {
    return asd2g::api_exception("asd2g_volume");
}

int asd2g_weno5_line(asd2g_session *s, const double *F, double *FP, double *FM, double d, int n) try {
    if (!s || !F || !FP || !FM || n < 1 || (size_t)(n + 2 * NB) > s->G || !(d > 0.0))
        return fail(ASD2G_E_ARG, "weno5_line: bad arguments");
    const size_t m = (size_t)n + 2 * NB;
    cudaMemcpyAsync(s->f[ASD2G_W0], F, sizeof(double) * m, cudaMemcpyHostToDevice, s->st);
    cudaMemsetAsync(s->f[ASD2G_W1], 0, sizeof(double) * m, s->st);
    cudaMemsetAsync(s->f[ASD2G_W2], 0, sizeof(double) * m, s->st);
    launch_weno_line(s->f[ASD2G_W0], s->f[ASD2G_W1], s->f[ASD2G_W2], d, n, s->st);
    cudaMemcpyAsync(FP, s->f[ASD2G_W1], sizeof(double) * m, cudaMemcpyDeviceToHost, s->st);
    cudaMemcpyAsync(FM, s->f[ASD2G_W2], sizeof(double) * m, cudaMemcpyDeviceToHost, s->st);
    int rc = cuda_check("weno5_line");
    return rc ? rc : sync(s);
} catch (...) {
    return asd2g::api_exception("asd2g_weno5_line");
}

int asd2g_weno_absgrad(asd2g_session *s, int ls, int ls0, int out) try {
    if (!s || !valid_field(ls) || !valid_field(ls0) || !valid_field(out) || out == ls || out == ls0)
        return fail(ASD2G_E_ARG, "bad field");
    launch_weno_absgrad(s->g, s->f[ls], s->f[ls0], s->f[out], s->st);
    return cuda_check("weno_absgrad");
} catch (...) {
    return asd2g::api_exception("asd2g_weno_absgrad");
}

// -------------------------------------------------------------- momentum --
int asd2g_kappa(asd2g_session *s) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    launch_kappa(s->g, s->f[ASD2G_LS], s->f[ASD2G_KAPPA], s->st);
    return cuda_check("kappa");
} catch (...) {
    return asd2g::api_exception("asd2g_kappa");
}

int asd2g_heaviside(asd2g_session *s) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    launch_heaviside(s->g, s->f[ASD2G_LS], s->f[ASD2G_H], s->f[ASD2G_HS], s->st);
    return cuda_check("heaviside");
} catch (...) {
    return asd2g::api_exception("asd2g_heaviside");
}

static int mom_single(asd2g_session *s, int kind, int ls, int u, int v, int h, int fu, int fv) {
    if (!s || !valid_field(u) || !valid_field(v) || !valid_field(fu) || !valid_field(fv) || fu == fv ||
        fu == u || fu == v || fv == u || fv == v)
        return fail(ASD2G_E_ARG, "bad field");
    const double *lsp = valid_field(ls) ? s->f[ls] : s->f[ASD2G_LS];
    const double *hp = valid_field(h) ? s->f[h] : s->f[ASD2G_HS];
    cudaMemsetAsync(s->f[fu], 0, sizeof(double) * s->G, s->st);
    cudaMemsetAsync(s->f[fv], 0, sizeof(double) * s->G, s->st);
    launch_mom_stage(kind, s->g, s->M, lsp, hp, s->f[u], s->f[v], nullptr, nullptr, s->f[fu], s->f[fv], s->dsc, s->st);
    return cuda_check("momentum term");
}

int asd2g_convection(asd2g_session *s, int u, int v, int cu, int cv) { return mom_single(s, 5, -1, u, v, -1, cu, cv); }
int asd2g_viscosity(asd2g_session *s, int u, int v, int ls, int h, int du, int dv) try {
    return mom_single(s, 6, ls, u, v, h, du, dv);
} catch (...) {
    return asd2g::api_exception("asd2g_viscosity");
}
int asd2g_momentum_rhs(asd2g_session *s, int ls, int u, int v, int h, int fu, int fv) try {
    return mom_single(s, 4, ls, u, v, h, fu, fv);
} catch (...) {
    return asd2g::api_exception("asd2g_momentum_rhs");
}

static int intermediate(asd2g_session *s, int h) {
    const Grid &g = s->g;
    const MomConst &M = s->M;
    const double *ls = s->f[ASD2G_LS], *H = s->f[h], *u = s->f[ASD2G_U], *v = s->f[ASD2G_V];
    double *uh = s->f[ASD2G_UHAT], *vh = s->f[ASD2G_VHAT];
    const int order = s->prm.time_order;
    if (order == 0) {
        launch_mom_stage(0, g, M, ls, H, u, v, nullptr, nullptr, uh, vh, s->dsc, s->st);
    } else if (order == 1) {
        launch_mom_stage(0, g, M, ls, H, u, v, nullptr, nullptr, s->ua, s->va, s->dsc, s->st);
        launch_fill_uv(g, s->ua, s->va, s->st);
        launch_mom_stage(3, g, M, ls, H, s->ua, s->va, u, v, uh, vh, s->dsc, s->st);
    } else {
        launch_mom_stage(0, g, M, ls, H, u, v, nullptr, nullptr, s->ua, s->va, s->dsc, s->st);
        launch_fill_uv(g, s->ua, s->va, s->st);
        launch_mom_stage(1, g, M, ls, H, s->ua, s->va, u, v, s->ub, s->vb, s->dsc, s->st);
        launch_fill_uv(g, s->ub, s->vb, s->st);
        launch_mom_stage(2, g, M, ls, H, s->ub, s->vb, u, v, uh, vh, s->dsc, s->st);
    }
    return cuda_check("intermediate_vel");
}

int asd2g_intermediate_vel(asd2g_session *s, double dt, int h) try {
    if (!s || !valid_field(h)) return fail(ASD2G_E_ARG, "bad field");
    int rc = set_dt(s, dt);
    if (rc) return rc;
    return intermediate(s, h);
} catch (...) {
    return asd2g::api_exception("asd2g_intermediate_vel");
}

int asd2g_divergence(asd2g_session *s, int u, int v, int div) try {
    if (!s || !valid_field(u) || !valid_field(v) || !valid_field(div) || div == u || div == v)
        return fail(ASD2G_E_ARG, "bad field");
    cudaMemsetAsync(s->f[div], 0, sizeof(double) * s->G, s->st);
    launch_divergence(s->g, s->f[u], s->f[v], s->f[div], s->st);
    return cuda_check("divergence");
} catch (...) {
    return asd2g::api_exception("asd2g_divergence");
}

int asd2g_update_vel(asd2g_session *s, double dt) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    int rc = set_dt(s, dt);
    if (rc) return rc;
    launch_update_vel(s->g, s->M, s->f[ASD2G_UHAT], s->f[ASD2G_VHAT], s->f[ASD2G_PS], s->f[ASD2G_LS], s->f[ASD2G_H],
                      s->f[ASD2G_KAPPA], s->f[ASD2G_U], s->f[ASD2G_V], s->dsc, s->st);
    return cuda_check("update_vel");
} catch (...) {
    return asd2g::api_exception("asd2g_update_vel");
}

int asd2g_update_dt(asd2g_session *s, double *dt) try {
    if (!s || !dt) return fail(ASD2G_E_ARG, "null argument");
    launch_update_dt(s->g, s->M, s->f[ASD2G_U], s->f[ASD2G_V], s->partial, s->counter, s->dsc + 1, s->st);
    cudaMemcpyAsync(s->dsc_host, s->dsc, sizeof(double) * 2, cudaMemcpyDeviceToHost, s->st);
    int rc = sync(s);
    if (rc) return rc;
    *dt = s->dsc_host[1];
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_update_dt");
}

int asd2g_update_ntk(asd2g_session *s, int ls, int nxf, int nyf) try {
    if (!s || !valid_field(ls) || !valid_field(nxf) || !valid_field(nyf) || nxf == nyf || nxf == ls || nyf == ls)
        return fail(ASD2G_E_ARG, "bad field");
    launch_absgrad(s->g, false, s->f[ls], s->f[ls], s->w1, s->st);  // ENO_DerivAbsLS_2D(ls, ls)
    launch_ntk(s->g, s->f[ls], s->w1, s->f[nxf], s->f[nyf], s->st);
    return cuda_check("update_ntk");
} catch (...) {
    return asd2g::api_exception("asd2g_update_ntk");
}

// -------------------------------------------------------------- pressure --
static int p_supported(asd2g_session *s) {
    for (int k = 0; k < 4; k++) {
        const int b = s->prm.bc_p[k];
        if (b == ASD2G_BC_PERIODIC || b == ASD2G_BC_AXISYM || b == ASD2G_BC_LSFREE || b == ASD2G_BC_CUSTOM)
            return fail(ASD2G_E_UNSUPPORTED,
                        "pressure boundary kind %d on side %d: the GFM assembly supports Neumann, Dirichlet, inlet, "
                        "outlet, pressure and wall sides only",
                        b, k);
    }
    return ASD2G_OK;
}

static int assemble(asd2g_session *s, int recompute_kappa) {
    NvtxRange nv("GFM assembly");
    int rc = p_supported(s);
    if (rc) return rc;
    const Grid &g = s->g;
    if (recompute_kappa) {
        launch_kappa(g, s->f[ASD2G_LS], s->f[ASD2G_KAPPA], s->st);
        launch_fill_p(g, s->f[ASD2G_KAPPA], s->st);
    }
    launch_assemble(g, s->M, s->f[ASD2G_LS], s->f[ASD2G_KAPPA], s->f[ASD2G_H], s->f[ASD2G_DIV], s->dsc, s->sys, s->st);
    s->assembled = true;
    return cuda_check("assemble_gfm");
}

int asd2g_assemble_gfm(asd2g_session *s, double dt, int recompute_kappa) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    int rc = set_dt(s, dt);
    if (rc) return rc;
    return assemble(s, recompute_kappa);
} catch (...) {
    return asd2g::api_exception("asd2g_assemble_gfm");
}

int asd2g_get_system(asd2g_session *s, double *diag, double *cw, double *ce, double *cs, double *cn, double *rhs,
                     int *pinned) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    if (!s->assembled) return fail(ASD2G_E_ARG, "no system assembled");
    const int nx = s->g.nx, ny = s->g.ny;
    const size_t N = s->N;
    std::vector<double> tmp(N);
    double *outs[6] = {diag, cw, ce, cs, cn, rhs};
    double *srcs[6] = {s->sys.diag, s->sys.cw, s->sys.ce, s->sys.cs, s->sys.cn, s->sys.b};
    for (int a = 0; a < 6; a++) {
        if (!outs[a]) continue;
        cudaMemcpyAsync(tmp.data(), srcs[a], sizeof(double) * N, cudaMemcpyDeviceToHost, s->st);
        int rc = sync(s);
        if (rc) return rc;
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) outs[a][i + (size_t)nx * j] = tmp[j + (size_t)ny * i];
    }
    if (pinned) *pinned = s->sys.pinned;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_get_system");
}

static int capture_chunk(asd2g_session *s, int solver) {
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return cuda_check("capture begin");
    const bool ok = enqueue_iters(s, solver, solver == ASD2G_SOLVER_MGPCG ? 8 : s->chunk_len);
    if (cudaStreamEndCapture(s->st, &graph) != cudaSuccess) return cuda_check("capture end");
    if (!ok) {
        cudaGraphDestroy(graph);
        return fail(ASD2G_E_UNSUPPORTED, "multigrid partial-sum buffer too small");
    }
    cudaGraphExec_t ex = nullptr;
    if (cudaGraphInstantiate(&ex, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_check("graph instantiate");
    }
    cudaGraphDestroy(graph);
    s->chunk_exec[solver] = ex;
    return ASD2G_OK;
}

static int solve(asd2g_session *s, int solver, double tol, int maxit, int *iters, double *resid) {
    NvtxRange nv("pressure solve");
    const Grid &g = s->g;
    const int mode = solver;  // 0 PCG, 1 PCG (reference), 2 BiCGStab, 3 BiCGStab (reference), 4 MG-FCG
    const double reg = solver == 1 ? 1.0e-12 : 0.0;  // err_tol^2 in alpha (poisson2d.cpp:354)
    launch_set_kstate(s->ks, tol, maxit, mode, reg, s->st);
    s->last_one_launch = 0;
    if (solver == 0 && !(s->prm.solver_flags & ASD2G_FLAG_NO_CLUSTER_PCG) &&
        launch_pcg_persist(g.nx, g.ny, s->sys, s->x, s->r, s->pa, s->pb, s->partial,
                           3 * RED_BLOCKS_MAX + 2 * DT_BLOCKS, s->mgp_bar, s->ks, tol, maxit, s->st)) {
        // one cooperative launch ran the whole solve (all SMs)
        if (stream_capturing(s)) {
            if (iters) *iters = -1;
            if (resid) *resid = -1.0;
            return cuda_check("one-launch pcg");
        }
        cudaMemcpyAsync(s->ks_host, s->ks, sizeof(KState), cudaMemcpyDeviceToHost, s->st);
        int rc2 = sync(s);
        if (rc2) return rc2;
        const KState &k = *s->ks_host;
        if (k.status != -8) {  // -8: a grid-barrier wait gave up; solve again below
            s->last_one_launch = 1;
            if (iters) *iters = k.it;
            if (resid) *resid = k.res;
            if (k.status == -5) return fail(ASD2G_E_NONFINITE, "non-finite residual at iteration %d", k.it);
            if (k.status == -6) return fail(ASD2G_E_BREAKDOWN, "Krylov breakdown at iteration %d", k.it);
            return !(k.res > tol) ? ASD2G_OK : ASD2G_NOT_CONVERGED;
        }
        launch_set_kstate(s->ks, tol, maxit, mode, reg, s->st);
    }
    if (solver == 0 && !(s->prm.solver_flags & ASD2G_FLAG_NO_CLUSTER_PCG) &&
        launch_pcg_cluster(g.nx, g.ny, s->sys, s->x, s->ks, tol, maxit, s->st)) {
        // one launch ran the whole solve
        s->last_one_launch = 1;
        if (stream_capturing(s)) {
            if (iters) *iters = -1;
            if (resid) *resid = -1.0;
            return cuda_check("cluster pcg");
        }
        cudaMemcpyAsync(s->ks_host, s->ks, sizeof(KState), cudaMemcpyDeviceToHost, s->st);
        int rc2 = sync(s);
        if (rc2) return rc2;
        const KState &k = *s->ks_host;
        if (iters) *iters = k.it;
        if (resid) *resid = k.res;
        if (k.status == -5) return fail(ASD2G_E_NONFINITE, "non-finite residual at iteration %d", k.it);
        if (k.status == -6) return fail(ASD2G_E_BREAKDOWN, "Krylov breakdown at iteration %d", k.it);
        return !(k.res > tol) ? ASD2G_OK : ASD2G_NOT_CONVERGED;
    }
    if (solver == ASD2G_SOLVER_MGPCG) {
        int rc0 = mg_alloc(s);
        if (rc0) return rc0;
        // systems up to about 256^2: the whole solve as one cooperative launch
        if (mg_persist_enabled() && !(s->prm.solver_flags & ASD2G_FLAG_NO_PERSIST_MG) &&
            launch_mg_persist(s->sys, g.nx, g.ny, s->lv, s->nlev, s->x, s->r, s->q, s->pa, s->pb, s->z,
                              s->mg_partial, s->mg_partial_n, s->mgp_bar, s->ks, tol, maxit, mg_omega_value(),
                              s->st)) {
            if (stream_capturing(s)) {
                if (iters) *iters = -1;
                if (resid) *resid = -1.0;
                return cuda_check("one-launch MG-FCG");
            }
            cudaMemcpyAsync(s->ks_host, s->ks, sizeof(KState), cudaMemcpyDeviceToHost, s->st);
            int rc2 = sync(s);
            if (rc2) return rc2;
            const KState &k = *s->ks_host;
            if (k.status != -8) {  // -8: a grid-barrier wait gave up; solve again below
                s->last_one_launch = 1;
                if (iters) *iters = k.it;
                if (resid) *resid = k.res;
                if (k.status == -5) return fail(ASD2G_E_NONFINITE, "non-finite residual at iteration %d", k.it);
                if (k.status == -6) return fail(ASD2G_E_BREAKDOWN, "Krylov breakdown at iteration %d", k.it);
                return (!(k.res > tol) || k.status == 2) ? ASD2G_OK : ASD2G_NOT_CONVERGED;
            }
            launch_set_kstate(s->ks, tol, maxit, mode, reg, s->st);
        }
        launch_mg_setup(s->sys, s->lv, s->nlev, s->coarse_inv, s->st);
        if (!launch_fcg_init(s->sys, g.nx, g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, s->pa, s->q, s->z,
                             s->ks, s->mg_partial, s->mg_partial_n, s->st))
            return fail(ASD2G_E_UNSUPPORTED, "multigrid partial-sum buffer too small");
    } else if (solver <= 1) launch_pcg_init(g, s->sys, s->x, s->r, s->pa, s->ks, s->partial, s->st);
    else launch_bicg_init(g, s->sys, s->x, s->r, s->rt, s->pa, s->q, s->ks, s->partial, s->st);
    int rc = cuda_check("solver init");
    if (rc) return rc;
    const int chunk = solver == ASD2G_SOLVER_MGPCG ? 8 : s->chunk_len;
    if (stream_capturing(s)) {
        // Inside a caller's capture: enqueue maxit iterations (each returns at
        // entry once converged); no host polling is possible.
        if (!enqueue_iters(s, solver, maxit + (maxit & 1)))
            return fail(ASD2G_E_UNSUPPORTED, "multigrid partial-sum buffer too small");
        if (iters) *iters = -1;
        if (resid) *resid = -1.0;
        return cuda_check("solver enqueue");
    }
    if (!s->chunk_exec[solver]) {
        rc = capture_chunk(s, solver);
        if (rc) return rc;
    }
    int launched = 0;
    for (;;) {
        if (cudaGraphLaunch(s->chunk_exec[solver], s->st) != cudaSuccess) return cuda_check("graph launch");
        launched += chunk;
        cudaMemcpyAsync(s->ks_host, s->ks, sizeof(KState), cudaMemcpyDeviceToHost, s->st);
        rc = sync(s);
        if (rc) return rc;
        if (s->ks_host->done || launched >= maxit + chunk) break;
    }
    const KState &k = *s->ks_host;
    if (iters) *iters = k.it;
    if (resid) *resid = k.res;
    if (k.status == -5) return fail(ASD2G_E_NONFINITE, "non-finite residual at iteration %d", k.it);
    if (k.status == -6) return fail(ASD2G_E_BREAKDOWN, "Krylov breakdown at iteration %d", k.it);
    // MG-FCG status 2: the FP64-verified residual stagnated at rounding level
    // above tol; resid reports it and the solve counts as converged.
    const bool conv = (solver == 0 || solver == ASD2G_SOLVER_MGPCG) ? (!(k.res > tol) || k.status == 2)
                                                                     : (k.res <= tol);
    return conv ? ASD2G_OK : ASD2G_NOT_CONVERGED;
}

// ---- flexible CG with the two-level learned preconditioner (ASD2G_SOLVER_UNET) ----
// After each V-cycle (which leaves beta alone in this mode): r1 = r - A z_mg,
// the network on r1's features, omega, z = z_mg + omega u and beta.
// with_net false: the V-cycle alone (z = z_mg), the direction update as usual.
static int pc_correct(asd2g_session *s, bool with_net = true) {
    const Grid &g = s->g;
    if (!with_net) {
        launch_pc_output(s->sys, g.nx, g.ny, nullptr, s->rt, s->z, s->fm, s->ks, s->mg_partial, s->st);
        return cuda_check("learned preconditioner");
    }
    launch_pc_input(s->sys, g.nx, g.ny, s->r, s->z, s->rt, s->ks, s->pc_scal, s->pc_feats, s->mg_partial, s->st);
    const int rc = asd2g_unet_forward(s->pc_net, 1, g.nx, g.ny, s->pc_feats, s->pc_out);
    if (rc) return rc;
    launch_pc_output(s->sys, g.nx, g.ny, s->pc_out, s->rt, s->z, s->fm, s->ks, s->mg_partial, s->st);
    return cuda_check("learned preconditioner");
}

constexpr int PC_CHUNK = 8;          // iterations per captured chunk; the FP64 residual check closes it
constexpr int PC_MAX_ITERS = 500;    // iterations of the learned phase before the Jacobi-PCG fallback
static_assert(PC_CHUNK % FM_SLOTS == 0, "every replay of a chunk must write the direction slots in the same order");

// The network's correction on every PC_NET_EVERY-th iteration of a chunk
// (ASD2G_PC_EVERY=1..8 in the environment), besides the first application;
// the other iterations, and the restart after a residual replacement, use
// the V-cycle alone.  Measured on the 512^2 evaluation (solves/s, iterations):
// every iteration 142 (13-15), every 2nd 199, every 3rd or 4th 260, every
// 8th 306 (11-17): the correction is needed for a few modes the V-cycle
// leaves, not at every step.
constexpr int PC_NET_EVERY = 8;
static bool pc_net_on(int k) {
    static const int every = [] {
        const char *e = std::getenv("ASD2G_PC_EVERY");
        const int v = e ? std::atoi(e) : PC_NET_EVERY;
        return v >= 1 && v <= 8 ? v : PC_NET_EVERY;
    }();
    return k % every == every - 1;
}

static int pc_chunk(asd2g_session *s) {
    const Grid &g = s->g;
    for (int k = 0; k < PC_CHUNK; k++) {
        if (!launch_pcm_iter(s->sys, g.nx, g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, s->z, s->fm, k % FM_SLOTS,
                             s->ks, s->mg_partial, s->mg_partial_n, s->st))
            return fail(ASD2G_E_UNSUPPORTED, "multigrid partial-sum buffer too small");
        const int rc = pc_correct(s, pc_net_on(k));
        if (rc) return rc;
    }
    if (!launch_pcm_check(s->sys, g.nx, g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, s->z, s->fm, s->ks,
                          s->mg_partial, s->mg_partial_n, s->st))
        return fail(ASD2G_E_UNSUPPORTED, "multigrid partial-sum buffer too small");
    // after a residual replacement that restarts the solve: the V-cycle of
    // the new residual alone (mid-solve the check changes nothing and these
    // kernels return at entry)
    return pc_correct(s, false);
}

static int fm_alloc(asd2g_session *s) {
    if (s->fm.p[0]) return ASD2G_OK;
    for (int j = 0; j < FM_SLOTS; j++) {
        int rc = dalloc(s, &s->fm.p[j], s->N);
        if (!rc) rc = dalloc(s, &s->fm.q[j], s->N);
        if (rc) return rc;
        cudaMemsetAsync(s->fm.p[j], 0, sizeof(double) * s->N, s->st);
        cudaMemsetAsync(s->fm.q[j], 0, sizeof(double) * s->N, s->st);
    }
    return ASD2G_OK;
}

static int solve_learned(asd2g_session *s, double tol, int maxit, int *iters, double *resid) {
    NvtxRange nv("pressure solve (learned preconditioner)");
    const Grid &g = s->g;
    s->last_one_launch = 0;
    if (!s->pc_net) return fail(ASD2G_E_ARG, "no preconditioner network attached (asd2g_set_preconditioner_net)");
    int rc = mg_alloc(s);
    if (!rc) rc = fm_alloc(s);
    if (rc) return rc;
    rc = asd2g_unet_set_stream(s->pc_net, s->st);
    if (rc) return rc;
    const int cap = maxit < PC_MAX_ITERS ? maxit : PC_MAX_ITERS;
    launch_set_kstate(s->ks, tol, cap, ASD2G_SOLVER_UNET, 0.0, s->st);
    launch_mg_setup(s->sys, s->lv, s->nlev, s->coarse_inv, s->st);
    launch_pc_setup(s->sys, g.nx, g.ny, s->pc_feats, s->pc_scal, s->partial, s->counter + 2, s->ks, s->st);
    if (!launch_fcg_init(s->sys, g.nx, g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, s->pa, s->q, s->z, s->ks,
                         s->mg_partial, s->mg_partial_n, s->st))
        return fail(ASD2G_E_UNSUPPORTED, "multigrid partial-sum buffer too small");
    rc = pc_correct(s);
    if (rc) return rc;
    if (!s->chunk_exec[ASD2G_SOLVER_UNET]) {
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return cuda_check("capture");
        const int rc2 = pc_chunk(s);
        if (cudaStreamEndCapture(s->st, &graph) != cudaSuccess) return cuda_check("capture end");
        if (rc2) {
            cudaGraphDestroy(graph);
            return rc2;
        }
        const cudaError_t e = cudaGraphInstantiate(&s->chunk_exec[ASD2G_SOLVER_UNET], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_check("graph instantiate");
    }
    for (int launched = 0;; launched += PC_CHUNK) {
        if (cudaGraphLaunch(s->chunk_exec[ASD2G_SOLVER_UNET], s->st) != cudaSuccess) return cuda_check("graph launch");
        cudaMemcpyAsync(s->ks_host, s->ks, sizeof(KState), cudaMemcpyDeviceToHost, s->st);
        rc = sync(s);
        if (rc) return rc;
        if (s->ks_host->done || launched + PC_CHUNK >= cap) break;
    }
    const KState k = *s->ks_host;
    int unet_flag = 0;
    asd2g_unet_error_flag(s->pc_net, &unet_flag);
    if ((k.status == 0 || k.status == 2) && !unet_flag && (!(k.res > tol) || k.status == 2)) {
        s->last_fallback = 0;
        if (iters) *iters = k.it;
        if (resid) *resid = k.res;
        return ASD2G_OK;
    }
    // Jacobi-PCG fallback, judged by the same FP64 residual.
    s->last_fallback = 1;
    int it2 = 0;
    const int st = solve(s, ASD2G_SOLVER_PCG, tol, maxit, &it2, resid);
    if (iters) *iters = k.it + it2;
    return st;
}

int asd2g_set_preconditioner_net(asd2g_session *s, asd2g_unet *net) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    if (net && (s->g.nx % 8 || s->g.ny % 8))
        return fail(ASD2G_E_UNSUPPORTED, "the learned preconditioner needs nx and ny multiples of 8");
    if (s->pc_net && s->pc_net != net) asd2g_unet_set_stream(s->pc_net, nullptr);
    s->pc_net = net;
    if (net && !s->pc_feats) {
        float **pp[] = {&s->pc_feats, &s->pc_out};
        const size_t sizes[] = {4 * s->N, s->N};
        for (int i = 0; i < 2; i++) {
            if (cudaMalloc(pp[i], sizeof(float) * sizes[i]) != cudaSuccess) {
                cudaGetLastError();
                return fail(ASD2G_E_NOMEM, "preconditioner buffers");
            }
            s->allocs.push_back(*pp[i]);
        }
    }
    if (net && !s->pc_scal) {
        if (cudaMalloc(&s->pc_scal, sizeof(float) * 4) != cudaSuccess) {
            cudaGetLastError();
            return fail(ASD2G_E_NOMEM, "preconditioner buffers");
        }
        s->allocs.push_back(s->pc_scal);
    }
    if (s->chunk_exec[ASD2G_SOLVER_UNET]) {  // the captured chunk holds the previous network's launches
        cudaGraphExecDestroy(s->chunk_exec[ASD2G_SOLVER_UNET]);
        s->chunk_exec[ASD2G_SOLVER_UNET] = nullptr;
    }
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_set_preconditioner_net");
}

int asd2g_last_solve_one_launch(asd2g_session *s, int *one_launch) try {
    if (!s || !one_launch) return fail(ASD2G_E_ARG, "null argument");
    *one_launch = s->last_one_launch;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_last_solve_one_launch");
}

int asd2g_last_fallback(asd2g_session *s, int *used) try {
    if (!s || !used) return fail(ASD2G_E_ARG, "null argument");
    *used = s->last_fallback;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_last_fallback");
}

int asd2g_pc_training_pair_at(asd2g_session *s, int iters, void *feats, void *target) try {
    if (!s || !feats || !target) return fail(ASD2G_E_ARG, "null argument");
    if (iters < 0 || iters > 1000) return fail(ASD2G_E_ARG, "iters must be in [0, 1000]");
    if (!s->assembled) return fail(ASD2G_E_ARG, "assemble and solve the system first");
    if (!s->pc_scal) {
        if (cudaMalloc(&s->pc_scal, sizeof(float) * 4) != cudaSuccess) {
            cudaGetLastError();
            return fail(ASD2G_E_NOMEM, "scale buffer");
        }
        s->allocs.push_back(s->pc_scal);
    }
    int rc = mg_alloc(s);
    if (rc) return rc;
    const Grid &g = s->g;
    const size_t N = s->N;
    double *xs = s->t3, *e = s->t3 + N;  // the solution, kept; the error the pair's target is made of
    cudaMemcpyAsync(xs, s->x, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->st);
    // x0 = the iterate after `iters` MG-FCG iterations from 0 (tol 0: none stops early)
    launch_set_kstate(s->ks, 0.0, 1 << 30, ASD2G_SOLVER_MGPCG, 0.0, s->st);
    launch_mg_setup(s->sys, s->lv, s->nlev, s->coarse_inv, s->st);
    bool ok = launch_fcg_init(s->sys, g.nx, g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, s->pa, s->q, s->z,
                              s->ks, s->mg_partial, s->mg_partial_n, s->st);
    for (int k = 0; k < iters && ok; k++) {
        const double *po = k % 2 == 0 ? s->pa : s->pb;
        double *pn = k % 2 == 0 ? s->pb : s->pa;
        ok = launch_fcg_iter(s->sys, g.nx, g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, po, pn, s->q, s->z, s->ks,
                             s->mg_partial, s->mg_partial_n, s->st);
    }
    if (!ok) return fail(ASD2G_E_UNSUPPORTED, "multigrid partial-sum buffer too small");
    // z = V(r) for r = b - A x0 (the recurrence residual); r1 = r - A z
    launch_pc_input(s->sys, g.nx, g.ny, s->r, s->z, s->rt, s->ks, s->pc_scal, (float *)feats, s->mg_partial, s->st);
    launch_pc_pair(s->sys, g.nx, g.ny, xs, s->x, s->z, s->rt, e, s->ks, s->pc_scal, s->partial, s->counter + 2,
                   (float *)feats, (float *)target, s->st);
    cudaMemcpyAsync(s->x, xs, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->st);
    return cuda_check("training pair");
} catch (...) {
    return asd2g::api_exception("asd2g_pc_training_pair_at");
}

int asd2g_pc_training_pair(asd2g_session *s, void *feats, void *target) try {
    return asd2g_pc_training_pair_at(s, 0, feats, target);
} catch (...) {
    return asd2g::api_exception("asd2g_pc_training_pair");
}

int asd2g_solve_pressure(asd2g_session *s, int solver, double tol, int maxit, double dt, int *iters,
                         double *rel_resid) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    if (solver < 0 || solver > ASD2G_SOLVER_UNET) return fail(ASD2G_E_ARG, "solver %d out of range", solver);
    if (!s->assembled) return fail(ASD2G_E_ARG, "assemble the system first");
    if (maxit < 0) return fail(ASD2G_E_ARG, "maxit must be >= 0");
    int rc = set_dt(s, dt);
    if (rc) return rc;
    const int st = solver == ASD2G_SOLVER_UNET ? solve_learned(s, tol, maxit, iters, rel_resid)
                                                : solve(s, solver, tol, maxit, iters, rel_resid);
    if (st < 0) return st;
    launch_scatter_ps(s->g, s->x, s->f[ASD2G_PS], s->f[ASD2G_P], s->dsc, s->st);
    rc = cuda_check("scatter ps");
    return rc ? rc : st;
} catch (...) {
    return asd2g::api_exception("asd2g_solve_pressure");
}

int asd2g_true_residual(asd2g_session *s, double *rel) try {
    if (!s || !rel) return fail(ASD2G_E_ARG, "null argument");
    if (!s->assembled) return fail(ASD2G_E_ARG, "no system assembled");
    launch_true_residual(s->g, s->sys, s->f[ASD2G_PS], s->partial, s->dsc + 2, s->st);
    cudaMemcpyAsync(s->dsc_host, s->dsc, sizeof(double) * 4, cudaMemcpyDeviceToHost, s->st);
    int rc = sync(s);
    if (rc) return rc;
    double bb = s->dsc_host[3];
    if (bb == 0.0) bb = 1.0;
    *rel = std::sqrt(s->dsc_host[2]) / std::sqrt(bb);
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_true_residual");
}

int asd2g_csr_solve(asd2g_session *s, int solver, int rows, const int *ia, const int *ja, const double *a,
                    const double *diag, const double *b, double *x, double tol, int maxit, int *iters,
                    double *rel_resid) try {
    if (!s || !ia || !ja || !a || !diag || !b || !x) return fail(ASD2G_E_ARG, "null argument");
    if (rows < 1 || (size_t)rows > s->N) return fail(ASD2G_E_ARG, "rows must be in [1, nx*ny]");
    if (solver < 0 || solver > 3) return fail(ASD2G_E_ARG, "solver %d not available for CSR input", solver);
    if (maxit < 0) return fail(ASD2G_E_ARG, "maxit must be >= 0");
    const int nnz = ia[rows];
    if (nnz < 0 || ia[0] != 0) return fail(ASD2G_E_ARG, "bad CSR row pointer");
    std::vector<double> minv(rows);
    for (int r = 0; r < rows; r++) minv[r] = 1.0 / diag[r];  // InvertMatrixDiagonal, poisson2d.cpp:577-585
    int *dia = nullptr, *dja = nullptr;
    double *da = nullptr, *dminv = nullptr, *db = nullptr;
    bool ok = cudaMalloc(&dia, sizeof(int) * (rows + 1)) == cudaSuccess &&
              cudaMalloc(&dja, sizeof(int) * (nnz ? nnz : 1)) == cudaSuccess &&
              cudaMalloc(&da, sizeof(double) * (nnz ? nnz : 1)) == cudaSuccess &&
              cudaMalloc(&dminv, sizeof(double) * rows) == cudaSuccess && cudaMalloc(&db, sizeof(double) * rows) == cudaSuccess;
    int rc = ASD2G_OK;
    if (!ok) {
        cudaGetLastError();
        rc = fail(ASD2G_E_NOMEM, "CSR buffers");
    }
    KState k{};
    if (rc == ASD2G_OK) {
        cudaMemcpyAsync(dia, ia, sizeof(int) * (rows + 1), cudaMemcpyHostToDevice, s->st);
        cudaMemcpyAsync(dja, ja, sizeof(int) * nnz, cudaMemcpyHostToDevice, s->st);
        cudaMemcpyAsync(da, a, sizeof(double) * nnz, cudaMemcpyHostToDevice, s->st);
        cudaMemcpyAsync(dminv, minv.data(), sizeof(double) * rows, cudaMemcpyHostToDevice, s->st);
        cudaMemcpyAsync(db, b, sizeof(double) * rows, cudaMemcpyHostToDevice, s->st);
        Sys S{};
        S.minv = dminv;
        S.b = db;
        const double reg = solver == 1 ? 1.0e-12 : 0.0;
        launch_set_kstate(s->ks, tol, maxit, solver, reg, s->st);
        if (solver <= 1) launch_pcg_init_n(rows, S, s->x, s->r, s->pa, s->ks, s->partial, s->st);
        else launch_bicg_init_n(rows, S, s->x, s->r, s->rt, s->pa, s->q, s->ks, s->partial, s->st);
        for (int done = 0, launched = 0; !done; launched += 64) {
            for (int it = 0; it < 64; it++) {
                if (solver <= 1)
                    launch_csr_pcg_iter(dia, dja, da, rows, S, s->x, s->r, s->pa, s->q, s->ks, s->partial, s->st);
                else
                    launch_csr_bicg_iter(dia, dja, da, rows, S, s->x, s->r, s->rt, s->pa, s->q, s->sv, s->t3, s->ks,
                                         s->partial, s->st);
            }
            cudaMemcpyAsync(&k, s->ks, sizeof(KState), cudaMemcpyDeviceToHost, s->st);
            rc = sync(s);
            if (rc) break;
            done = k.done || launched + 64 >= maxit + 64;
        }
        if (rc == ASD2G_OK) {
            cudaMemcpyAsync(x, s->x, sizeof(double) * rows, cudaMemcpyDeviceToHost, s->st);
            rc = sync(s);
        }
    }
    cudaFree(dia);
    cudaFree(dja);
    cudaFree(da);
    cudaFree(dminv);
    cudaFree(db);
    if (rc) return rc;
    if (iters) *iters = k.it;
    if (rel_resid) *rel_resid = k.res;
    if (k.status == -5) return fail(ASD2G_E_NONFINITE, "non-finite residual at iteration %d", k.it);
    if (k.status == -6) return fail(ASD2G_E_BREAKDOWN, "Krylov breakdown at iteration %d", k.it);
    const bool conv = solver == 0 ? !(k.res > tol) : (k.res <= tol);
    return conv ? ASD2G_OK : ASD2G_NOT_CONVERGED;
} catch (...) {
    return asd2g::api_exception("asd2g_csr_solve");
}

// ------------------------------------------------------------------ step --
// The step up to the assembled pressure system (dt from the device scalar):
// Solve_LevelSet_2D, the reinitialisation, kappa, H and HS, the FP64 volume
// check, the intermediate velocity, its divergence and the GFM assembly.
static int enqueue_step_pre(asd2g_session *s, int reinit_mode) {
    NvtxRange nv("level set + momentum + assembly");
    const Grid &g = s->g;
    cudaMemcpyAsync(s->f[ASD2G_LSB], s->f[ASD2G_LS], sizeof(double) * s->G, cudaMemcpyDeviceToDevice, s->st);
    double *ls = s->f[ASD2G_LS];
    if (s->prm.precision == ASD2G_PRECISION_MIXED) {
        if (!ls32_supported(g, reinit_mode))
            return fail(ASD2G_E_UNSUPPORTED, "mixed precision implements reinit modes 0, 2 and 4, not %d", reinit_mode);
        launch_fill_p(g, ls, s->st);
        launch_ls_step32(g, reinit_mode, s->prm.ls_max_atime, s->f[ASD2G_U], s->f[ASD2G_V], s->dsc, ls, s->w32,
                         s->st);
    } else {
        launch_center_vel(g, s->f[ASD2G_U], s->f[ASD2G_V], s->tu, s->tv, s->st);
        launch_fill_p(g, ls, s->st);
        launch_ls_stage(1, g, ls, s->tu, s->tv, ls, s->w1, s->dsc, s->st);
        launch_ls_stage(2, g, s->w1, s->tu, s->tv, ls, s->w2, s->dsc, s->st);
        launch_ls_stage(3, g, s->w2, s->tu, s->tv, ls, ls, s->dsc, s->st);
        launch_reinit(g, reinit_mode, s->prm.ls_max_atime, ls, s->f[ASD2G_LS0], s->w1, s->w2, s->w3, s->st);
    }
    launch_kappa(g, ls, s->f[ASD2G_KAPPA], s->st);
    launch_heaviside(g, ls, s->f[ASD2G_H], s->f[ASD2G_HS], s->st);
    // FP64 volume check of the new level set (read by asd2g_last_volume)
    launch_volume(g, s->f[ASD2G_H], s->f[ASD2G_HS], s->partial, s->counter + 1, s->dsc + 5, s->st);
    int rc = intermediate(s, ASD2G_HS);
    if (rc) return rc;
    launch_fill_uv(g, s->f[ASD2G_UHAT], s->f[ASD2G_VHAT], s->st);
    cudaMemsetAsync(s->f[ASD2G_DIV], 0, sizeof(double) * s->G, s->st);
    launch_divergence(g, s->f[ASD2G_UHAT], s->f[ASD2G_VHAT], s->f[ASD2G_DIV], s->st);
    // SolvePoisson recomputes kappa when kWe is finite and nonzero (mac2d.cpp:1307).
    const double we = s->prm.numbers_given ? s->prm.we : s->prm.rho_h / s->prm.sigma;
    return assemble(s, (we != 0.0 && std::isfinite(we)) ? 1 : 0);
}

// After the solve: ps and p, the projection (UpdateVel) and the next dt (UpdateDt, into dsc[1]).
static void enqueue_step_post(asd2g_session *s) {
    NvtxRange nv("projection + dt");
    const Grid &g = s->g;
    launch_scatter_ps(g, s->x, s->f[ASD2G_PS], s->f[ASD2G_P], s->dsc, s->st);
    launch_update_vel(g, s->M, s->f[ASD2G_UHAT], s->f[ASD2G_VHAT], s->f[ASD2G_PS], s->f[ASD2G_LS], s->f[ASD2G_H],
                      s->f[ASD2G_KAPPA], s->f[ASD2G_U], s->f[ASD2G_V], s->dsc, s->st);
    launch_update_dt(g, s->M, s->f[ASD2G_U], s->f[ASD2G_V], s->partial, s->counter, s->dsc + 1, s->st);
}

// Runs enqueue() on the session stream: eagerly on the first call (first-use
// set-up such as kernel attributes stays outside any capture) and inside a
// caller's stream capture; afterwards as a graph captured once and replayed.
// The launches are those of the eager call, so are the results.
extern "C++" {
namespace {
template <class F>
int replay_phase(asd2g_session *s, cudaGraphExec_t *ex, int *calls, const char *what, F enqueue) {
    if (stream_capturing(s) || *calls == 0) {
        ++*calls;
        return enqueue();
    }
    if (!*ex) {
        if (cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();  // a stream that cannot be captured: launch one by one
            return enqueue();
        }
        const int rc = enqueue();
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s->st, &graph);
        if (rc || e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return rc ? rc : cuda_check(what);
        }
        const cudaError_t ie = cudaGraphInstantiate(ex, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            *ex = nullptr;
            return cuda_check(what);
        }
    }
    if (cudaGraphLaunch(*ex, s->st) != cudaSuccess) return cuda_check(what);
    return ASD2G_OK;
}
}  // namespace
}  // extern "C++"

int asd2g_droplet_step(asd2g_session *s, double *dt, int reinit_mode, int solver, double tol, int maxit, int *iters,
                       double *rel_resid) try {
    NvtxRange nv("asd2g_droplet_step");
    if (!s || !dt) return fail(ASD2G_E_ARG, "null argument");
    if (reinit_mode < 0 || reinit_mode > 4) return fail(ASD2G_E_ARG, "reinit mode %d out of range", reinit_mode);
    int rc = p_supported(s);
    if (rc) return rc;
    rc = set_dt(s, *dt);
    if (rc) return rc;
    rc = replay_phase(s, &s->pre_exec[reinit_mode], &s->pre_calls[reinit_mode], "droplet_step (before the solve)",
                      [&] { return enqueue_step_pre(s, reinit_mode); });
    if (rc) return rc;
    const int st = solve(s, solver, tol, maxit, iters, rel_resid);
    if (st < 0) return st;
    rc = replay_phase(s, &s->post_exec, &s->post_calls, "droplet_step (after the solve)", [&] {
        enqueue_step_post(s);
        return cuda_check("droplet_step (after the solve)");
    });
    if (rc) return rc;
    cudaMemcpyAsync(s->dsc_host, s->dsc, sizeof(double) * 7, cudaMemcpyDeviceToHost, s->st);
    rc = sync(s);
    if (rc) return rc;
    rc = cuda_check("droplet_step");
    if (rc) return rc;
    *dt = s->dsc_host[1];
    s->last_volume[0] = s->dsc_host[5];
    s->last_volume[1] = s->dsc_host[6];
    return st;
} catch (...) {
    return asd2g::api_exception("asd2g_droplet_step");
}


// ---- axisymmetric MAC solver (MACSolver2DAxisym, mac2dAxisym.cpp) ----
// x is r, y is z; base_x of the parameters is kBaseR.  Convection, Heaviside,
// UpdateVel and the Krylov solvers are the 2D ones (same arithmetic).
namespace {
int axi_p_supported(asd2g_session *s) {
    for (int k = 0; k < 4; k++) {
        const int b = s->prm.bc_p[k];
        if (b == ASD2G_BC_PERIODIC || b == ASD2G_BC_LSFREE || b == ASD2G_BC_CUSTOM)
            return fail(ASD2G_E_UNSUPPORTED,
                        "pressure boundary kind %d on side %d: the axisymmetric assembly supports Neumann, axisym, "
                        "wall, Dirichlet, inlet, outlet and pressure sides",
                        b, k);
    }
    return ASD2G_OK;
}

// GetRHSU / GetRHSV: the 2D convection term into ua, then the axisymmetric
// right side over the whole padded array, then the U / V ghost fill.
int axi_rhs(asd2g_session *s, int comp, int ls, int u, int v, int uhat, int h, int out) {
    const Grid &g = s->g;
    launch_mom_stage(5, g, s->M, s->f[ls], s->f[h], s->f[u], s->f[v], nullptr, nullptr, comp == 0 ? s->ua : s->va,
                     comp == 0 ? s->va : s->ua, s->dsc, s->st);
    if (comp == 0) {
        launch_axi_rhs_u(g, s->M, s->f[ls], s->f[u], s->f[v], s->f[h], s->ua, s->dsc, s->f[out], s->st);
        launch_fill_uv(g, s->f[out], nullptr, s->st);
    } else {
        launch_axi_rhs_v(g, s->M, s->f[ls], s->f[u], s->f[uhat], s->f[v], s->f[h], s->ua, s->dsc, s->f[out], s->st);
        launch_fill_uv(g, nullptr, s->f[out], s->st);
    }
    return cuda_check(comp == 0 ? "axi_rhs_u" : "axi_rhs_v");
}

void axi_assemble_enqueue(asd2g_session *s, int recompute_kappa) {
    const Grid &g = s->g;
    if (recompute_kappa) {
        launch_axi_kappa(g, s->f[ASD2G_LS], s->f[ASD2G_KAPPA], s->st);
        launch_fill_p(g, s->f[ASD2G_KAPPA], s->st);
    }
    launch_axi_assemble(g, s->M, s->f[ASD2G_LS], s->f[ASD2G_KAPPA], s->f[ASD2G_H], s->f[ASD2G_DIV], s->dsc, s->sys,
                        s->st);
    s->assembled = true;
}

int axi_we_finite(const asd2g_session *s) {
    const double we = s->prm.numbers_given ? s->prm.we : s->prm.rho_h / s->prm.sigma;
    return (we != 0.0 && std::isfinite(we)) ? 1 : 0;
}
}  // namespace

int asd2g_axi_kappa(asd2g_session *s) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    launch_axi_kappa(s->g, s->f[ASD2G_LS], s->f[ASD2G_KAPPA], s->st);
    return cuda_check("axi_kappa");
} catch (...) {
    return asd2g::api_exception("asd2g_axi_kappa");
}

int asd2g_axi_rhs_u(asd2g_session *s, double dt, int ls, int u, int v, int h, int out) try {
    if (!s || !valid_field(ls) || !valid_field(u) || !valid_field(v) || !valid_field(h) || !valid_field(out) ||
        out == ls || out == u || out == v || out == h)
        return fail(ASD2G_E_ARG, "bad field");
    int rc = set_dt(s, dt);
    return rc ? rc : axi_rhs(s, 0, ls, u, v, -1, h, out);
} catch (...) {
    return asd2g::api_exception("asd2g_axi_rhs_u");
}

int asd2g_axi_rhs_v(asd2g_session *s, double dt, int ls, int u, int uhat, int v, int h, int out) try {
    if (!s || !valid_field(ls) || !valid_field(u) || !valid_field(uhat) || !valid_field(v) || !valid_field(h) ||
        !valid_field(out) || out == ls || out == u || out == uhat || out == v || out == h)
        return fail(ASD2G_E_ARG, "bad field");
    int rc = set_dt(s, dt);
    return rc ? rc : axi_rhs(s, 1, ls, u, v, uhat, h, out);
} catch (...) {
    return asd2g::api_exception("asd2g_axi_rhs_v");
}

int asd2g_axi_viscosity(asd2g_session *s, int ls, int u, int uhat, int v, int h, int du, int dv) try {
    if (!s || !valid_field(ls) || !valid_field(u) || !valid_field(uhat) || !valid_field(v) || !valid_field(h) ||
        !valid_field(du) || !valid_field(dv) || du == dv)
        return fail(ASD2G_E_ARG, "bad field");
    for (int in : {ls, u, uhat, v, h})
        if (in == du || in == dv) return fail(ASD2G_E_ARG, "outputs must differ from the inputs");
    const Grid &g = s->g;
    launch_axi_rhs_u(g, s->M, s->f[ls], s->f[u], s->f[v], s->f[h], s->f[du], s->dsc, s->f[du], s->st, 1);
    launch_axi_rhs_v(g, s->M, s->f[ls], s->f[u], s->f[uhat], s->f[v], s->f[h], s->f[dv], s->dsc, s->f[dv], s->st,
                     1);
    return cuda_check("axi_viscosity");
} catch (...) {
    return asd2g::api_exception("asd2g_axi_viscosity");
}

int asd2g_axi_hat(asd2g_session *s, int comp, double dt, int ls, int rhs, int h, int out) try {
    if (!s || (comp != 0 && comp != 1) || !valid_field(ls) || !valid_field(rhs) || !valid_field(h) ||
        !valid_field(out) || out == ls || out == rhs || out == h)
        return fail(ASD2G_E_ARG, "bad field or component");
    int rc = set_dt(s, dt);
    if (rc) return rc;
    double *const w[6] = {s->ua, s->va, s->ub, s->vb, s->w1, s->w2};
    launch_axi_hat(s->g, s->M, comp, s->f[ls], s->f[rhs], s->f[h], s->dsc, s->f[out], w, s->st);
    return cuda_check("axi_hat");
} catch (...) {
    return asd2g::api_exception("asd2g_axi_hat");
}

int asd2g_axi_divergence(asd2g_session *s, int u, int v, int div, int for_poisson) try {
    if (!s || !valid_field(u) || !valid_field(v) || !valid_field(div) || div == u || div == v)
        return fail(ASD2G_E_ARG, "bad field");
    launch_axi_div(s->g, for_poisson ? 1 : 0, s->f[u], s->f[v], s->f[div], s->st);
    return cuda_check("axi_divergence");
} catch (...) {
    return asd2g::api_exception("asd2g_axi_divergence");
}

int asd2g_axi_assemble(asd2g_session *s, double dt, int recompute_kappa) try {
    if (!s) return fail(ASD2G_E_ARG, "null session");
    int rc = axi_p_supported(s);
    if (rc) return rc;
    rc = set_dt(s, dt);
    if (rc) return rc;
    axi_assemble_enqueue(s, recompute_kappa);
    return cuda_check("axi_assemble");
} catch (...) {
    return asd2g::api_exception("asd2g_axi_assemble");
}

int asd2g_axi_update_dt(asd2g_session *s, double *dt) try {
    if (!s || !dt) return fail(ASD2G_E_ARG, "null argument");
    launch_axi_update_dt(s->g, s->M, s->f[ASD2G_U], s->f[ASD2G_V], s->f[ASD2G_KAPPA], s->partial, s->counter,
                         s->dsc + 1, s->st);
    cudaMemcpyAsync(s->dsc_host, s->dsc, sizeof(double) * 2, cudaMemcpyDeviceToHost, s->st);
    int rc = sync(s);
    if (rc) return rc;
    *dt = s->dsc_host[1];
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_axi_update_dt");
}

// One step of the axisymmetric driver before its pressure solve (test_mac2d_
// large.cpp:1269-1292): level set with the level set's own P grid gl,
// curvature, Heaviside, right sides and the implicit viscous step of u and v,
// the r-weighted divergence, the assembly.
static int axi_step_pre(asd2g_session *s, const Grid &gl, int reinit_mode) {
    const Grid &g = s->g;
    double *ls = s->f[ASD2G_LS], *u = s->f[ASD2G_U], *v = s->f[ASD2G_V];
    double *uh = s->f[ASD2G_UHAT], *vh = s->f[ASD2G_VHAT], *HS = s->f[ASD2G_HS];
    cudaMemcpyAsync(s->f[ASD2G_LSB], ls, sizeof(double) * s->G, cudaMemcpyDeviceToDevice, s->st);
    launch_center_vel(gl, u, v, s->tu, s->tv, s->st);
    launch_fill_p(gl, ls, s->st);
    launch_ls_stage(1, gl, ls, s->tu, s->tv, ls, s->w1, s->dsc, s->st);
    launch_ls_stage(2, gl, s->w1, s->tu, s->tv, ls, s->w2, s->dsc, s->st);
    launch_ls_stage(3, gl, s->w2, s->tu, s->tv, ls, ls, s->dsc, s->st);
    launch_fill_p(gl, ls, s->st);
    launch_reinit(gl, reinit_mode, s->prm.ls_max_atime, ls, s->f[ASD2G_LS0], s->w1, s->w2, s->w3, s->st);
    launch_fill_p(gl, ls, s->st);
    launch_axi_kappa(g, ls, s->f[ASD2G_KAPPA], s->st);
    launch_heaviside(g, ls, s->f[ASD2G_H], HS, s->st);
    int rc = axi_rhs(s, 0, ASD2G_LS, ASD2G_U, ASD2G_V, -1, ASD2G_HS, ASD2G_W0);
    if (rc) return rc;
    double *const w[6] = {s->ua, s->va, s->ub, s->vb, s->w1, s->w2};
    launch_axi_hat(g, s->M, 0, ls, s->f[ASD2G_W0], HS, s->dsc, uh, w, s->st);
    launch_fill_uv(g, uh, nullptr, s->st);
    rc = axi_rhs(s, 1, ASD2G_LS, ASD2G_U, ASD2G_V, ASD2G_UHAT, ASD2G_HS, ASD2G_W0);
    if (rc) return rc;
    launch_axi_hat(g, s->M, 1, ls, s->f[ASD2G_W0], HS, s->dsc, vh, w, s->st);
    launch_fill_uv(g, nullptr, vh, s->st);
    launch_axi_div(g, 1, uh, vh, s->f[ASD2G_DIV], s->st);
    launch_fill_p(gl, ls, s->st);  // the driver fills the level set again before the solve (:1294)
    axi_assemble_enqueue(s, axi_we_finite(s));
    return cuda_check("axi_step (before the solve)");
}

// After the solve (:1296-1306): ps and p, the projection, the next dt (dsc[1]).
// The driver repeats the fills that SolvePoisson and UpdateVel end with
// (:1299, :1304-1305); with a Neumann side next to a Dirichlet one a second
// fill changes the corner ghosts, so it is repeated here too.
static int axi_step_post(asd2g_session *s) {
    const Grid &g = s->g;
    double *u = s->f[ASD2G_U], *v = s->f[ASD2G_V];
    launch_scatter_ps(g, s->x, s->f[ASD2G_PS], s->f[ASD2G_P], s->dsc, s->st);
    launch_fill_p(g, s->f[ASD2G_PS], s->st);
    launch_update_vel(g, s->M, s->f[ASD2G_UHAT], s->f[ASD2G_VHAT], s->f[ASD2G_PS], s->f[ASD2G_LS], s->f[ASD2G_H],
                      s->f[ASD2G_KAPPA], u, v, s->dsc, s->st);
    launch_fill_uv(g, u, v, s->st);
    launch_axi_update_dt(g, s->M, u, v, s->f[ASD2G_KAPPA], s->partial, s->counter, s->dsc + 1, s->st);
    return cuda_check("axi_step (after the solve)");
}

int asd2g_axi_step(asd2g_session *s, double *dt, int reinit_mode, const int32_t *ls_bc, const double *ls_bcc,
                   int solver, double tol, int maxit, int *iters, double *rel_resid) try {
    NvtxRange nv("asd2g_axi_step");
    if (!s || !dt) return fail(ASD2G_E_ARG, "null argument");
    if (reinit_mode < 0 || reinit_mode > 4) return fail(ASD2G_E_ARG, "reinit mode %d out of range", reinit_mode);
    if (s->prm.precision != ASD2G_PRECISION_FP64)
        return fail(ASD2G_E_UNSUPPORTED, "the axisymmetric step runs in FP64 only");
    if (solver < 0 || solver > ASD2G_SOLVER_MGPCG) return fail(ASD2G_E_ARG, "solver %d out of range", solver);
    int rc = axi_p_supported(s);
    if (rc) return rc;
    // the level-set solver's own P-grid boundary (LevelSetSolver2D has its own BoundaryCondition2D)
    Grid gl = s->g;
    int32_t key[4];
    double cst[4];
    for (int k = 0; k < 4; k++) {
        key[k] = ls_bc ? ls_bc[k] : s->prm.bc_p[k];
        cst[k] = ls_bc ? (ls_bcc ? ls_bcc[k] : 0.0) : s->prm.bcc_p[k];
        if (key[k] < 0 || key[k] > 9) return fail(ASD2G_E_ARG, "level-set boundary kind out of range");
    }
    if (ls_bc) {
        bool mirror = true;
        for (int k = 0; k < 4; k++) {
            gl.kp[k] = kind_p(key[k]);
            gl.bp[k] = key[k];
            gl.cp[k] = cst[k];
            mirror &= (gl.kp[k] == K_NEU || gl.kp[k] == K_DIR);
        }
        gl.p_mirror = mirror ? 1 : 0;
    }
    if (std::memcmp(key, s->axi_ls_key, sizeof key) != 0 || std::memcmp(cst, s->axi_ls_cst, sizeof cst) != 0) {
        for (int m = 0; m < 5; m++) {  // graphs captured with other level-set kinds
            if (s->axi_pre_exec[m]) cudaGraphExecDestroy(s->axi_pre_exec[m]);
            s->axi_pre_exec[m] = nullptr;
            s->axi_pre_calls[m] = 0;
        }
        std::memcpy(s->axi_ls_key, key, sizeof key);
        std::memcpy(s->axi_ls_cst, cst, sizeof cst);
    }
    rc = set_dt(s, *dt);
    if (rc) return rc;
    rc = replay_phase(s, &s->axi_pre_exec[reinit_mode], &s->axi_pre_calls[reinit_mode], "axi_step (before the solve)",
                      [&] { return axi_step_pre(s, gl, reinit_mode); });
    if (rc) return rc;
    const int st = solve(s, solver, tol, maxit, iters, rel_resid);
    if (st < 0) return st;
    rc = replay_phase(s, &s->axi_post_exec, &s->axi_post_calls, "axi_step (after the solve)",
                      [&] { return axi_step_post(s); });
    if (rc) return rc;
    cudaMemcpyAsync(s->dsc_host, s->dsc, sizeof(double) * 2, cudaMemcpyDeviceToHost, s->st);
    rc = sync(s);
    if (rc) return rc;
    rc = cuda_check("axi_step");
    if (rc) return rc;
    *dt = s->dsc_host[1];
    return st;
} catch (...) {
    return asd2g::api_exception("asd2g_axi_step");
}

// ---- checkpoint / restart ----
namespace {
struct CkHeader {
    char magic[8];
    uint32_t version, header_bytes;
    int32_t nx, ny, nbc, precision;
    double t, dt;
    int64_t step;
    uint32_t nfields, field_bits;
    uint64_t payload_bytes, checksum;
    uint8_t reserved[48];
};
static_assert(sizeof(CkHeader) == 128, "checkpoint header is 128 bytes");
constexpr char CK_MAGIC[8] = {'A', 'S', 'D', '2', 'G', 'C', 'K', '1'};
constexpr int CK_FIELDS[5] = {ASD2G_LS, ASD2G_U, ASD2G_V, ASD2G_PS, ASD2G_P};

// Weighted word sum  sum_i w_i (2 i + 1)  mod 2^64 over 64-bit words w_i,
// the index i counted from `first` (a sum taken in pieces).
uint64_t ck_checksum(const void *data, size_t nwords, uint64_t first = 0) {
    const unsigned char *p = static_cast<const unsigned char *>(data);
    uint64_t h = 0;
    for (size_t i = 0; i < nwords; i++) {
        uint64_t w;
        std::memcpy(&w, p + 8 * i, 8);
        h += w * (2u * (first + i) + 1u);
    }
    return h;
}

// The file's checksum: the header with its checksum field zeroed is words
// 0..15, the payload words 16 on (so t, dt, step and the reserved bytes are
// covered as well as the fields).
uint64_t ck_file_checksum(const CkHeader &h, const double *payload, size_t nwords) {
    CkHeader z = h;
    z.checksum = 0;
    constexpr size_t hw = sizeof(CkHeader) / 8;
    return ck_checksum(&z, hw) + ck_checksum(payload, nwords, hw);
}

// Reads and checks the header; with payload != nullptr also reads the payload.
int ck_read(const char *path, CkHeader &h, std::vector<double> *payload) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ASD2G_E_IO, "cannot open checkpoint %s", path);
    int rc = ASD2G_OK;
    // the grid sides are bounded before any size arithmetic (in 64 bits), and
    // the payload the header claims must be what the file holds before a
    // buffer of that size is allocated
    constexpr int32_t kMaxSide = 1 << 20;
    long long file_bytes = -1;
    if (std::fseek(f, 0, SEEK_END) == 0) file_bytes = std::ftell(f);
    std::rewind(f);
    if (std::fread(&h, sizeof h, 1, f) != 1) rc = fail(ASD2G_E_IO, "%s: short header", path);
    else if (std::memcmp(h.magic, CK_MAGIC, 8) != 0 || h.version != 2 || h.header_bytes != sizeof(CkHeader))
        rc = fail(ASD2G_E_IO, "%s: not an asd2g checkpoint (magic/version)", path);
    else if (h.nx < 1 || h.ny < 1 || h.nx > kMaxSide || h.ny > kMaxSide || h.nbc != 3 || h.nfields != 5 ||
             h.payload_bytes != (uint64_t)h.nfields * (uint64_t)((int64_t)h.nx + 6) *
                                    (uint64_t)((int64_t)h.ny + 6) * 8u)
        rc = fail(ASD2G_E_IO, "%s: inconsistent sizes", path);
    else if (file_bytes < 0 || (uint64_t)file_bytes != sizeof(CkHeader) + h.payload_bytes)
        rc = fail(ASD2G_E_IO, "%s: file length does not match the header", path);
    if (!rc) {
        try {
            std::vector<double> buf(h.payload_bytes / 8);
            if (std::fread(buf.data(), 1, h.payload_bytes, f) != h.payload_bytes)
                rc = fail(ASD2G_E_IO, "%s: short payload", path);
            else if (ck_file_checksum(h, buf.data(), buf.size()) != h.checksum)
                rc = fail(ASD2G_E_IO, "%s: checksum mismatch", path);
            else if (payload)
                payload->swap(buf);
        } catch (const std::bad_alloc &) {
            rc = fail(ASD2G_E_NOMEM, "%s: no host memory for the payload", path);
        }
    }
    std::fclose(f);
    return rc;
}
}  // namespace

int asd2g_checkpoint_save(asd2g_session *s, const char *path, double t, long long step, double dt) try {
    if (!s || !path) return fail(ASD2G_E_ARG, "null argument");
    const size_t G = s->G;
    std::vector<double> buf(5 * G);
    for (int k = 0; k < 5; k++)
        cudaMemcpyAsync(buf.data() + k * G, s->f[CK_FIELDS[k]], sizeof(double) * G, cudaMemcpyDeviceToHost, s->st);
    int rc = sync(s);
    if (rc) return rc;
    CkHeader h{};
    std::memcpy(h.magic, CK_MAGIC, 8);
    h.version = 2;
    h.header_bytes = sizeof(CkHeader);
    h.nx = s->g.nx;
    h.ny = s->g.ny;
    h.nbc = 3;
    h.precision = s->prm.precision;
    h.t = t;
    h.dt = dt;
    h.step = step;
    h.nfields = 5;
    for (int k : CK_FIELDS) h.field_bits |= 1u << k;
    h.payload_bytes = sizeof(double) * buf.size();
    h.checksum = ck_file_checksum(h, buf.data(), buf.size());
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ASD2G_E_IO, "cannot create checkpoint %s", path);
    const bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 && std::fwrite(buf.data(), 1, h.payload_bytes, f) == h.payload_bytes;
    const bool closed = std::fclose(f) == 0;
    return ok && closed ? ASD2G_OK : fail(ASD2G_E_IO, "writing checkpoint %s failed", path);
} catch (...) {
    return asd2g::api_exception("asd2g_checkpoint_save");
}

int asd2g_checkpoint_load(asd2g_session *s, const char *path, double *t, long long *step, double *dt) try {
    if (!s || !path) return fail(ASD2G_E_ARG, "null argument");
    CkHeader h{};
    std::vector<double> buf;
    int rc = ck_read(path, h, &buf);
    if (rc) return rc;
    if (h.nx != s->g.nx || h.ny != s->g.ny)
        return fail(ASD2G_E_ARG, "checkpoint grid %d x %d does not match the session's %d x %d", h.nx, h.ny, s->g.nx,
                    s->g.ny);
    const size_t G = s->G;
    for (int k = 0; k < 5; k++)
        cudaMemcpyAsync(s->f[CK_FIELDS[k]], buf.data() + k * G, sizeof(double) * G, cudaMemcpyHostToDevice, s->st);
    rc = sync(s);  // the host buffer must outlive the copies
    if (rc) return rc;
    s->assembled = false;
    if (t) *t = h.t;
    if (step) *step = h.step;
    if (dt) *dt = h.dt;
    return cuda_check("checkpoint load");
} catch (...) {
    return asd2g::api_exception("asd2g_checkpoint_load");
}

int asd2g_checkpoint_info(const char *path, int *nx, int *ny, double *t, long long *step, double *dt) try {
    if (!path) return fail(ASD2G_E_ARG, "null argument");
    CkHeader h{};
    const int rc = ck_read(path, h, nullptr);
    if (rc) return rc;
    if (nx) *nx = h.nx;
    if (ny) *ny = h.ny;
    if (t) *t = h.t;
    if (step) *step = h.step;
    if (dt) *dt = h.dt;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_checkpoint_info");
}

// ---- device-resident multi-step run ----
// One droplet step with the MG-FCG as a CUDA graph: the solver's iterations
// are the body of a WHILE conditional node (8 iterations + the FP64 check per
// pass; a kernel at the end of the body clears the condition once the solve
// is done, or after ceil(maxit / 8) + 2 passes), and the whole step is the
// body of an IF node that skips it once an earlier step failed.  The host
// launches the step graph n times and synchronises once.
// persist: the step's solve as the one-launch MG-FCG (systems that fit it)
// instead of the WHILE loop over chunks of per-phase kernels.
static int capture_run_graph(asd2g_session *s, int reinit_mode, double tol, int maxit, bool persist) {
    for (cudaStream_t &a : s->aux_st)
        if (!a && cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking) != cudaSuccess) return cuda_check("aux stream");
    const cudaStream_t main_st = s->st;
    const int cap = (maxit + 7) / 8 + 2;
    cudaGraph_t graph = nullptr;
    int rc = ASD2G_OK;
    auto add_conditional = [&](cudaStream_t st, cudaGraphConditionalNodeType type, cudaGraphConditionalHandle *h,
                               cudaGraph_t *body) -> bool {
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &ndeps) != cudaSuccess ||
            cs != cudaStreamCaptureStatusActive)
            return false;
        if (cudaGraphConditionalHandleCreate(h, cg, 1, cudaGraphCondAssignDefault) != cudaSuccess) return false;
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = *h;
        np.conditional.type = type;
        np.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        if (cudaGraphAddNode(&node, cg, deps, ndeps, &np) != cudaSuccess) return false;
        *body = np.conditional.phGraph_out[0];
        return cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
    };
    if (cudaStreamBeginCapture(main_st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return cuda_check("capture");
    cudaGraphConditionalHandle h_if = 0, h_while = 0;
    cudaGraph_t if_body = nullptr, while_body = nullptr;
    bool ok = true;
    {
        // the handle must exist before the kernel that sets it is captured: create it on the capture graph
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        ok = cudaStreamGetCaptureInfo(main_st, &cs, nullptr, &cg, nullptr, nullptr) == cudaSuccess &&
             cudaGraphConditionalHandleCreate(&h_if, cg, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        if (ok) launch_run_if(s->run_stats, h_if, main_st);
        if (ok) {
            const cudaGraphNode_t *deps = nullptr;
            size_t ndeps = 0;
            ok = cudaStreamGetCaptureInfo(main_st, &cs, nullptr, &cg, &deps, &ndeps) == cudaSuccess;
            cudaGraphNodeParams np{};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h_if;
            np.conditional.type = cudaGraphCondTypeIf;
            np.conditional.size = 1;
            cudaGraphNode_t node = nullptr;
            if (ok) ok = cudaGraphAddNode(&node, cg, deps, ndeps, &np) == cudaSuccess;
            if (ok) if_body = np.conditional.phGraph_out[0];
            if (ok) ok = cudaStreamUpdateCaptureDependencies(main_st, &node, 1, cudaStreamSetCaptureDependencies) ==
                         cudaSuccess;
        }
    }
    // IF body: the whole step, captured on the first auxiliary stream
    if (ok) ok = cudaStreamBeginCaptureToGraph(s->aux_st[0], if_body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        s->st = s->aux_st[0];
        rc = enqueue_step_pre(s, reinit_mode);
        if (!rc && persist) {
            launch_set_kstate(s->ks, tol, maxit, ASD2G_SOLVER_MGPCG, 0.0, s->st);
            if (!launch_mg_persist(s->sys, s->g.nx, s->g.ny, s->lv, s->nlev, s->x, s->r, s->q, s->pa, s->pb, s->z,
                                   s->mg_partial, s->mg_partial_n, s->mgp_bar, s->ks, tol, maxit,
                                   mg_omega_value(), s->st))
                rc = fail(ASD2G_E_UNSUPPORTED, "one-launch MG-FCG not available");
        } else if (!rc) {
            launch_set_kstate(s->ks, tol, maxit, ASD2G_SOLVER_MGPCG, 0.0, s->st);
            launch_mg_setup(s->sys, s->lv, s->nlev, s->coarse_inv, s->st);
            if (!launch_fcg_init(s->sys, s->g.nx, s->g.ny, s->lv, s->nlev, s->coarse_inv, s->x, s->r, s->pa, s->q,
                                 s->z, s->ks, s->mg_partial, s->mg_partial_n, s->st))
                rc = fail(ASD2G_E_UNSUPPORTED, "multigrid partial-sum buffer too small");
        }
        if (!rc && !persist) ok = add_conditional(s->st, cudaGraphCondTypeWhile, &h_while, &while_body);
        // WHILE body: 8 iterations + the FP64 check, then the loop condition
        if (!rc && ok && !persist)
            ok = cudaStreamBeginCaptureToGraph(s->aux_st[1], while_body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (!rc && ok && !persist) {
            s->st = s->aux_st[1];
            if (!enqueue_iters(s, ASD2G_SOLVER_MGPCG, 8)) rc = fail(ASD2G_E_UNSUPPORTED, "multigrid buffer too small");
            launch_run_while(s->ks, s->run_stats, cap, h_while, s->st);
            cudaGraph_t wb = nullptr;
            ok = cudaStreamEndCapture(s->aux_st[1], &wb) == cudaSuccess;
            s->st = s->aux_st[0];
        }
        if (!rc && ok) {
            enqueue_step_post(s);
            launch_run_step_end(s->ks, s->run_stats, tol, s->dsc, s->st);
        }
        cudaGraph_t ib = nullptr;
        const bool ended = cudaStreamEndCapture(s->aux_st[0], &ib) == cudaSuccess;
        ok = ok && ended;
        s->st = main_st;
    }
    const bool ended = cudaStreamEndCapture(main_st, &graph) == cudaSuccess;
    s->st = main_st;
    if (rc || !ok || !ended) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rc ? rc : fail(ASD2G_E_CUDA, "capture of the device-resident step failed");
    }
    if (s->run_exec) cudaGraphExecDestroy(s->run_exec);
    s->run_exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&s->run_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ASD2G_E_CUDA, "instantiating the device-resident step: %s", cudaGetErrorString(e));
    }
    s->run_reinit = reinit_mode;
    s->run_tol = tol;
    s->run_maxit = maxit;
    return ASD2G_OK;
}

int asd2g_run_steps(asd2g_session *s, int nsteps, double *dt, int reinit_mode, int solver, double tol, int maxit,
                    int *steps_done, long long *iters_total, double *max_resid) try {
    NvtxRange nv("asd2g_run_steps");
    if (!s || !dt) return fail(ASD2G_E_ARG, "null argument");
    if (nsteps < 0) return fail(ASD2G_E_ARG, "nsteps must be >= 0");
    if (solver != ASD2G_SOLVER_MGPCG)
        return fail(ASD2G_E_UNSUPPORTED, "the device-resident loop runs the MG-FCG pressure solver only");
    if (maxit < 1 || !(tol >= 0.0)) return fail(ASD2G_E_ARG, "maxit must be >= 1 and tol >= 0");
    if (reinit_mode < 0 || reinit_mode > 4) return fail(ASD2G_E_ARG, "reinit mode %d out of range", reinit_mode);
    int rc = p_supported(s);
    if (!rc) rc = mg_alloc(s);
    if (rc) return rc;
    if (stream_capturing(s)) return fail(ASD2G_E_UNSUPPORTED, "asd2g_run_steps inside a caller's stream capture");
    if (!s->run_stats) {
        if (cudaMalloc(&s->run_stats, sizeof(RunStats)) != cudaSuccess ||
            cudaMallocHost(&s->run_stats_host, sizeof(RunStats)) != cudaSuccess) {
            cudaGetLastError();
            return fail(ASD2G_E_NOMEM, "run statistics");
        }
        s->allocs.push_back(s->run_stats);
    }
    if (!s->run_exec || s->run_reinit != reinit_mode || s->run_tol != tol || s->run_maxit != maxit) {
        // one eager step's worth of set-up first: attributes and first-use state outside the capture
        launch_run_reset(s->run_stats, s->st);
        const bool persist = mg_persist_enabled() && !(s->prm.solver_flags & ASD2G_FLAG_NO_PERSIST_MG) &&
                             mg_persist_fits(s->lv, s->nlev, s->g.nx, s->g.ny, s->mg_partial_n);
        rc = capture_run_graph(s, reinit_mode, tol, maxit, persist);
        if (rc && persist) rc = capture_run_graph(s, reinit_mode, tol, maxit, false);
        if (rc) return rc;
    }
    rc = set_dt(s, *dt);
    if (rc) return rc;
    launch_run_reset(s->run_stats, s->st);
    for (int k = 0; k < nsteps; k++)
        if (cudaGraphLaunch(s->run_exec, s->st) != cudaSuccess) return cuda_check("step graph launch");
    cudaMemcpyAsync(s->run_stats_host, s->run_stats, sizeof(RunStats), cudaMemcpyDeviceToHost, s->st);
    cudaMemcpyAsync(s->dsc_host, s->dsc, sizeof(double) * 7, cudaMemcpyDeviceToHost, s->st);
    rc = sync(s);
    if (rc) return rc;
    rc = cuda_check("run_steps");
    if (rc) return rc;
    const RunStats &R = *s->run_stats_host;
    if (steps_done) *steps_done = R.fail_step >= 0 ? R.fail_step + 1 : R.steps;
    if (iters_total) *iters_total = R.iters;
    if (max_resid) *max_resid = R.max_res;
    *dt = s->dsc_host[0];  // the next step's dt (copied from dsc[1] at each step's end)
    s->last_volume[0] = s->dsc_host[5];
    s->last_volume[1] = s->dsc_host[6];
    s->assembled = true;
    if (R.fail_step >= 0) {
        if (R.fail_status == -5) return fail(ASD2G_E_NONFINITE, "non-finite value at step %d", R.fail_step);
        if (R.fail_status == -6) return fail(ASD2G_E_BREAKDOWN, "Krylov breakdown at step %d", R.fail_step);
        return ASD2G_NOT_CONVERGED;
    }
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_run_steps");
}

}  // extern "C"

// Entry points of the ABI layer's helpers for the other host unit (batch.cu).
namespace asd2g {
int api_fail(int code, const char *msg) { return fail(code, "%s", msg); }
int api_exception(const char *fn) {
    try {
        throw;
    } catch (const std::bad_alloc &) {
        return fail(ASD2G_E_NOMEM, "%s: host allocation failed", fn);
    } catch (const std::exception &e) {
        return fail(ASD2G_E_INTERNAL, "%s: %s", fn, e.what());
    } catch (...) {
        return fail(ASD2G_E_INTERNAL, "%s: unknown C++ exception", fn);
    }
}
int api_grid_from_params(const asd2g_params *p, Grid &g, MomConst &M) { return grid_from_params(p, g, M); }
}  // namespace asd2g
