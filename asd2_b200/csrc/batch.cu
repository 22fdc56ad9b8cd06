// Batched GFM pressure solves (no reference counterpart: the reference solves
// one droplet per process).  A batch holds many droplet instances of uneven
// grid sizes; each phase -- assembly, multigrid set-up, every flexible-CG
// kernel, every V-cycle pass, the scatter -- is ONE kernel launch for the
// whole batch over device work lists of (instance, tile) or (instance, chunk)
// entries.  Each instance keeps its own solver scalars and stops on its own;
// chunks of iterations are captured once in a CUDA graph and replayed until
// every instance has converged.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "asd2g.h"
#include "batch.cuh"

namespace asd2g {
int api_fail(int code, const char *msg);
int api_exception(const char *fn);  // the entry points' exception handler (api.cu)
int api_grid_from_params(const asd2g_params *p, Grid &g, MomConst &M);
LsConst make_lsconst(const Grid &g);              // levelset.cu
template <typename T> LsConstT<T> make_lsconst_t(const Grid &g);
template <> LsConstT<float> make_lsconst_t<float>(const Grid &g);  // levelset32.cu
int reinit_steps(double adt, double max_atime);  // levelset.cu
}  // namespace asd2g

using namespace asd2g;

struct asd2g_batch {
    int count = 0;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    std::vector<asd2g_params> prm;
    std::vector<BInst> hinst;
    BInst *dinst = nullptr;
    std::vector<size_t> goff;  // padded-field offset of each instance
    size_t gtot = 0;
    double *pad = nullptr;     // BS_COUNT padded fields x gtot (BSlot order)
    double *sc = nullptr;      // 8 scalars per instance (BInst::sc)
    BTile *cell_tiles = nullptr;
    int ncell_tiles = 0;
    BatchPlan plan{};
    BStepPlan splan{};
    const BTile *shape_lists[MG_NSHAPES][MG_MAX_LEVELS] = {};  // uploaded tile lists per shape
    int shape_forced = -1;     // ASD2G_MG_TILE
    bool shape_tuned = false;  // the first solve timed every shape
    double shape_ms[MG_NSHAPES] = {};
    KState *ks = nullptr;
    KState *ks_host = nullptr;
    cudaGraphExec_t chunk_exec = nullptr;
    std::vector<void *> allocs;
    // learned preconditioner: the batch's own copy of the attached network,
    // and the instances grouped by grid size (one network pass per group,
    // whose feature planes are contiguous)
    struct PcGroup {
        int nx, ny, count;
        float *feats, *out;
    };
    asd2g_unet *net = nullptr;
    std::vector<PcGroup> groups;
    bool pc_ready = false;
    cudaGraphExec_t pc_exec = nullptr;
    int last_fallback = 0;
};

namespace {

constexpr int FCG_CHUNK_ITERS = 8;
constexpr int PAD_FIELDS = BS_COUNT;
constexpr int SC_PER_INST = 8;

int pad_slot(int field) {
    switch (field) {
    case ASD2G_LS: return BS_LS;
    case ASD2G_KAPPA: return BS_KAPPA;
    case ASD2G_H: return BS_H;
    case ASD2G_DIV: return BS_DIV;
    case ASD2G_PS: return BS_PS;
    case ASD2G_P: return BS_P;
    case ASD2G_U: return BS_U;
    case ASD2G_V: return BS_V;
    case ASD2G_HS: return BS_HS;
    case ASD2G_UHAT: return BS_UHAT;
    case ASD2G_VHAT: return BS_VHAT;
    case ASD2G_LSB: return BS_LSB;
    case ASD2G_LS0: return BS_LS0;
    default: return -1;
    }
}

template <typename T> int balloc(asd2g_batch *b, T **p, size_t n) {
    if (cudaMalloc(p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
        cudaGetLastError();
        return api_fail(ASD2G_E_NOMEM, "batch device allocation failed");
    }
    b->allocs.push_back(*p);
    return ASD2G_OK;
}

template <typename T> int upload_list(asd2g_batch *b, const std::vector<T> &v, const T **out) {
    T *d = nullptr;
    int rc = balloc(b, &d, v.size());
    if (rc) return rc;
    if (!v.empty()) cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, b->st);
    *out = d;
    return ASD2G_OK;
}

int check(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return ASD2G_OK;
    char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    return api_fail(ASD2G_E_CUDA, msg);
}

void release(asd2g_batch *b) {
    if (b->chunk_exec) cudaGraphExecDestroy(b->chunk_exec);
    if (b->pc_exec) cudaGraphExecDestroy(b->pc_exec);
    if (b->net) asd2g_unet_destroy(b->net);
    for (void *p : b->allocs) cudaFree(p);
    if (b->ks_host) cudaFreeHost(b->ks_host);
    if (b->own_stream && b->st) cudaStreamDestroy(b->st);
    delete b;
}

// Tile lists of the multigrid tile levels for MG_SHAPES[shape], and every
// instance's level-0 tile count (the ticket count of its level-0 dots).
int set_mg_shape(asd2g_batch *b, int shape) {
    const int ti = MG_SHAPES[shape][0], tj = MG_SHAPES[shape][1];
    std::vector<std::vector<BTile>> mgt(MG_MAX_LEVELS);
    for (int i = 0; i < b->count; i++) {
        BInst &I = b->hinst[i];
        for (int l = 0; l < I.s_cta; l++) {
            const int tx = (I.lv[l].ny + tj - 1) / tj, ty = (I.lv[l].nx + ti - 1) / ti;
            for (int by = 0; by < ty; by++)
                for (int bx = 0; bx < tx; bx++) mgt[l].push_back({i, bx, by});
        }
        I.tiles0 = ((I.lv[0].ny + tj - 1) / tj) * ((I.lv[0].nx + ti - 1) / ti);
    }
    BatchPlan &P = b->plan;
    int rc = ASD2G_OK;
    for (int l = 0; l < MG_MAX_LEVELS && !rc; l++) {
        if (b->shape_lists[shape][l] == nullptr && !mgt[l].empty())
            rc = upload_list(b, mgt[l], &b->shape_lists[shape][l]);
        P.mg_tiles[l] = b->shape_lists[shape][l];
        P.nmg_tiles[l] = (int)mgt[l].size();
    }
    if (rc) return rc;
    P.shape = shape;
    cudaMemcpyAsync(b->dinst, b->hinst.data(), sizeof(BInst) * b->count, cudaMemcpyHostToDevice, b->st);
    if (b->chunk_exec) {  // the captured chunk holds the previous shape's launches
        cudaGraphExecDestroy(b->chunk_exec);
        b->chunk_exec = nullptr;
    }
    return check("batch tile lists");
}

int build(asd2g_batch *b) {
    const int count = b->count;
    b->hinst.assign(count, BInst{});
    b->goff.assign(count, 0);
    std::vector<size_t> noff(count), poff(count);
    size_t ntot = 0, ptot = 0;
    std::vector<int> dims(2 * MG_MAX_LEVELS * (size_t)count);
    std::vector<size_t> mg_cells(MG_MAX_LEVELS, 0);
    for (int i = 0; i < count; i++) {
        BInst &I = b->hinst[i];
        int rc = api_grid_from_params(&b->prm[i], I.g, I.M);
        if (rc) return rc;
        if (!I.g.p_mirror)
            return api_fail(ASD2G_E_UNSUPPORTED, "batch instances need Neumann or Dirichlet pressure on all sides");
        I.dxx = make_divh(I.g.dx * I.g.dx);
        I.dyy = make_divh(I.g.dy * I.g.dy);
        I.n = (int64_t)I.g.nx * I.g.ny;
        I.chunks = (int)((I.n + FCG_CHUNK - 1) / FCG_CHUNK);
        I.tiles0 = batch_tiles0(I.g.nx, I.g.ny);
        I.nlev = mg_levels_for(I.g.nx, I.g.ny, &dims[2 * MG_MAX_LEVELS * (size_t)i], MG_MAX_LEVELS);
        if (I.nlev < 2) return api_fail(ASD2G_E_UNSUPPORTED, "instance too small for the multigrid preconditioner");
        b->goff[i] = b->gtot;
        b->gtot += (size_t)I.g.sx * I.g.sy;
        noff[i] = ntot;
        ntot += (size_t)I.n;
        poff[i] = ptot;
        ptot += (size_t)batch_partial_len(I.g.nx, I.g.ny);
        for (int l = 0; l < I.nlev; l++)
            mg_cells[l] += (size_t)dims[2 * MG_MAX_LEVELS * (size_t)i + 2 * l] * dims[2 * MG_MAX_LEVELS * (size_t)i + 2 * l + 1];
    }
    // arenas
    int rc = balloc(b, &b->pad, PAD_FIELDS * b->gtot);
    double *vec = nullptr, *partial = nullptr, *inv = nullptr;
    constexpr int NVEC = 13;  // diag cw ce cs cn minv b | x r pa pb q z
    if (!rc) rc = balloc(b, &vec, NVEC * ntot);
    if (!rc) rc = balloc(b, &partial, ptot);
    if (!rc) rc = balloc(b, &inv, (size_t)count * MG_COARSE_CELLS * MG_COARSE_CELLS);
    if (!rc) rc = balloc(b, &b->ks, (size_t)count);
    if (!rc) rc = balloc(b, &b->sc, (size_t)SC_PER_INST * count);
    std::vector<float *> mg_base(MG_MAX_LEVELS, nullptr);
    for (int l = 0; l < MG_MAX_LEVELS && !rc; l++)
        if (mg_cells[l]) rc = balloc(b, &mg_base[l], 6 * mg_cells[l]);
    if (rc) return rc;
    if (cudaMallocHost(&b->ks_host, sizeof(KState) * count) != cudaSuccess)
        return api_fail(ASD2G_E_NOMEM, "pinned allocation failed");
    cudaMemsetAsync(b->pad, 0, sizeof(double) * PAD_FIELDS * b->gtot, b->st);
    cudaMemsetAsync(vec, 0, sizeof(double) * NVEC * ntot, b->st);
    cudaMemsetAsync(b->sc, 0, sizeof(double) * SC_PER_INST * count, b->st);
    cudaMemsetAsync(b->ks, 0, sizeof(KState) * count, b->st);  // tickets start at 0
    std::vector<size_t> mg_used(MG_MAX_LEVELS, 0);
    for (int i = 0; i < count; i++) {
        BInst &I = b->hinst[i];
        const size_t go = b->goff[i], G = b->gtot;
        I.ls = b->pad + 0 * G + go;
        I.kappa = b->pad + 1 * G + go;
        I.H = b->pad + 2 * G + go;
        I.div = b->pad + 3 * G + go;
        I.ps = b->pad + 4 * G + go;
        I.p = b->pad + 5 * G + go;
        I.pad0 = b->pad + go;
        I.gstride = G;
        I.sc = b->sc + (size_t)SC_PER_INST * i;
        I.K = make_lsconst(I.g);
        I.ddx = make_divh(I.g.dx);
        I.ddy = make_divh(I.g.dy);
        I.d2x = make_divh(2.0 * I.g.dx);
        I.d2y = make_divh(2.0 * I.g.dy);
        const double hmin = I.g.dx < I.g.dy ? I.g.dx : I.g.dy;
        I.kappa_lim = 1.0 / hmin;
        I.hs_eps = hmin * 1.5;
        {
            const asd2g_params &pp = b->prm[i];
            const double we = pp.numbers_given ? pp.we : pp.rho_h / pp.sigma;
            I.kappa_fill = (we != 0.0 && std::isfinite(we)) ? 1 : 0;
            const double mt = pp.ls_max_atime > 0.0 ? pp.ls_max_atime : 1.5 * I.K.thick;
            I.nreinit = reinit_steps(I.K.adt, mt);
            I.order = pp.time_order;
        }
        double *v = vec + noff[i];
        double **slots[NVEC] = {&I.S.diag, &I.S.cw, &I.S.ce, &I.S.cs, &I.S.cn, &I.S.minv, &I.S.b,
                                &I.x, &I.r, &I.pa, &I.pb, &I.q, &I.z};
        for (int k = 0; k < NVEC; k++) *slots[k] = v + (size_t)k * ntot;
        I.S.pinned = I.g.pinned;
        I.ks = b->ks + i;
        I.partial = partial + poff[i];
        I.coarse_inv = inv + (size_t)i * MG_COARSE_CELLS * MG_COARSE_CELLS;
        const int *d = &dims[2 * MG_MAX_LEVELS * (size_t)i];
        for (int l = 0; l < I.nlev; l++) {
            MgLevel &L = I.lv[l];
            L.nx = d[2 * l];
            L.ny = d[2 * l + 1];
            const size_t m = (size_t)L.nx * L.ny, tot = mg_cells[l];
            float *base = mg_base[l] + mg_used[l];
            L.diag = base;
            L.ce = base + tot;
            L.cn = base + 2 * tot;
            L.f = base + 3 * tot;
            L.e = base + 4 * tot;
            L.ep = base + 5 * tot;
            mg_used[l] += m;
        }
        I.s_cta = mg_cta_first_level(I.lv, I.nlev);
    }
    for (int l = 0; l < MG_MAX_LEVELS; l++)
        if (mg_cells[l]) cudaMemsetAsync(mg_base[l], 0, sizeof(float) * 6 * mg_cells[l], b->st);
    // work lists
    // mixed instances: the FP32 level-set work arrays, each instance's start
    // rounded to 64 floats (paired FP32 accesses need 8-byte alignment)
    {
        size_t f32tot = 0;
        std::vector<size_t> f32off(count, 0);
        for (int i = 0; i < count; i++) {
            if (b->prm[i].precision != ASD2G_PRECISION_MIXED) continue;
            f32off[i] = f32tot;
            f32tot += ((size_t)b->hinst[i].g.sx * b->hinst[i].g.sy + 63) / 64 * 64;
        }
        float *f32 = nullptr;
        if (f32tot) {
            rc = balloc(b, &f32, (size_t)LS32_ARRAYS * f32tot);
            if (rc) return rc;
            cudaMemsetAsync(f32, 0, sizeof(float) * LS32_ARRAYS * f32tot, b->st);
        }
        for (int i = 0; i < count; i++) {
            BInst &I = b->hinst[i];
            I.mixed = b->prm[i].precision == ASD2G_PRECISION_MIXED ? 1 : 0;
            if (!I.mixed) continue;
            float *base = f32 + f32off[i];
            float **arr[LS32_ARRAYS] = {&I.w32.phi, &I.w32.ls0, &I.w32.a, &I.w32.b, &I.w32.tu, &I.w32.tv};
            for (int a = 0; a < LS32_ARRAYS; a++) *arr[a] = base + (size_t)a * f32tot;
            I.w32.band = nullptr;
            I.w32.band_n = nullptr;
            I.wk32 = make_weno32_const(I.g);
            I.K32 = make_lsconst_t<float>(I.g);
        }
    }
    std::vector<BTile> cells, s32, r32;
    std::vector<BChunk> chunks, padc, ghostc;
    std::vector<std::vector<BChunk>> lvl(MG_MAX_LEVELS);
    int max_s = 0, max_nlev = 0;
    for (int i = 0; i < count; i++) {
        const BInst &I = b->hinst[i];
        const int gx = (I.g.ny + TJ - 1) / TJ, gy = (I.g.nx + TI - 1) / TI;
        for (int by = 0; by < gy; by++)
            for (int bx = 0; bx < gx; bx++) cells.push_back({i, bx, by});
        for (int c = 0; c < I.chunks; c++) chunks.push_back({i, c});
        if (I.mixed) {  // FP32 strips: advection 64 columns x 16 rows, reinitialisation 60 x 8
            for (int by = 0; by < (I.g.nx + 15) / 16; by++)
                for (int bx = 0; bx < (I.g.ny + 63) / 64; bx++) s32.push_back({i, bx, by});
            for (int by = 0; by < (I.g.nx + 7) / 8; by++)
                for (int bx = 0; bx < (I.g.ny + 1 + 59) / 60; bx++) r32.push_back({i, bx, by});
        }
        const int64_t gi = (int64_t)I.g.sx * I.g.sy, ei = 2 * (int64_t)NB * (I.g.nx + I.g.ny);
        for (int c = 0; c < (int)((gi + BSTEP_PAD_CHUNK - 1) / BSTEP_PAD_CHUNK); c++) padc.push_back({i, c});
        for (int c = 0; c < (int)((ei + BSTEP_GHOST_CHUNK - 1) / BSTEP_GHOST_CHUNK); c++) ghostc.push_back({i, c});
        for (int l = 1; l < I.nlev; l++) {
            const int64_t m = (int64_t)I.lv[l].nx * I.lv[l].ny;
            for (int c = 0; c < (int)((m + FCG_CHUNK - 1) / FCG_CHUNK); c++) lvl[l].push_back({i, c});
        }
        max_s = I.s_cta > max_s ? I.s_cta : max_s;
        max_nlev = I.nlev > max_nlev ? I.nlev : max_nlev;
    }
    BatchPlan &P = b->plan;
    rc = balloc(b, &b->dinst, (size_t)count);
    if (rc) return rc;
    cudaMemcpyAsync(b->dinst, b->hinst.data(), sizeof(BInst) * count, cudaMemcpyHostToDevice, b->st);
    P.insts = b->dinst;
    P.count = count;
    const BTile *ct = nullptr;
    rc = upload_list(b, cells, &ct);
    b->cell_tiles = const_cast<BTile *>(ct);
    b->ncell_tiles = (int)cells.size();
    if (!rc) rc = upload_list(b, chunks, &P.chunks);
    P.nchunks = (int)chunks.size();
    for (int l = 0; l < MG_MAX_LEVELS && !rc; l++) {
        P.nlvl_chunks[l] = (int)lvl[l].size();
        if (!lvl[l].empty()) rc = upload_list(b, lvl[l], &P.lvl_chunks[l]);
    }
    P.max_s = max_s;
    P.max_nlev = max_nlev;
    const char *forced = std::getenv("ASD2G_MG_TILE");  // a fixed shape index (no tuning)
    b->shape_forced = forced && forced[0] >= '0' && forced[0] < '0' + MG_NSHAPES ? forced[0] - '0' : -1;
    if (!rc) rc = set_mg_shape(b, b->shape_forced >= 0 ? b->shape_forced : 0);
    BStepPlan &SP = b->splan;
    SP.insts = b->dinst;
    SP.count = count;
    SP.tiles = b->cell_tiles;
    SP.ntiles = b->ncell_tiles;
    SP.chunks = P.chunks;
    SP.nchunks = P.nchunks;
    if (!rc) rc = upload_list(b, padc, &SP.pad_chunks);
    SP.npad = (int)padc.size();
    if (!rc) rc = upload_list(b, ghostc, &SP.ghost_chunks);
    SP.nghost = (int)ghostc.size();
    SP.ns32 = (int)s32.size();
    SP.nr32 = (int)r32.size();
    SP.any_mixed = SP.ns32 > 0 ? 1 : 0;
    if (!rc && SP.ns32) rc = upload_list(b, s32, &SP.s32_tiles);
    if (!rc && SP.nr32) rc = upload_list(b, r32, &SP.r32_tiles);
    if (rc) return rc;
    if (!batch_cta_prepare()) return api_fail(ASD2G_E_CUDA, "coarse-cycle shared memory attribute");
    return check("batch set-up");
}

}  // namespace

extern "C" {

int asd2g_batch_create(const asd2g_params *params, int count, void *stream, asd2g_batch **out) try {
    if (!params || !out || count < 1) return api_fail(ASD2G_E_ARG, "batch_create: bad arguments");
    *out = nullptr;
    for (int i = 0; i < count; i++) {  // validate every instance before any device work
        Grid g{};
        MomConst M{};
        const int rc = api_grid_from_params(&params[i], g, M);
        if (rc) return rc;
        if (!g.p_mirror)
            return api_fail(ASD2G_E_UNSUPPORTED, "batch instances need Neumann or Dirichlet pressure on all sides");
    }
    asd2g_batch *b = new (std::nothrow) asd2g_batch();
    if (!b) return api_fail(ASD2G_E_NOMEM, "host allocation failed");
    b->count = count;
    b->prm.assign(params, params + count);
    if (stream) b->st = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess) {
            delete b;
            return api_fail(ASD2G_E_CUDA, "cudaStreamCreate failed");
        }
        b->own_stream = true;
    }
    const int rc = build(b);
    if (rc) {
        release(b);
        return rc;
    }
    *out = b;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_create");
}

int asd2g_batch_destroy(asd2g_batch *b) try {
    if (!b) return ASD2G_OK;
    cudaStreamSynchronize(b->st);
    release(b);
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_destroy");
}

int asd2g_batch_upload(asd2g_batch *b, int inst, int field, const double *host) try {
    const int slot = pad_slot(field);
    if (!b || !host || inst < 0 || inst >= b->count || slot < 0)
        return api_fail(ASD2G_E_ARG, "batch_upload: bad instance or field (LS, KAPPA, H, DIV, PS, P)");
    const Grid &g = b->hinst[inst].g;
    double *dst = b->pad + (size_t)slot * b->gtot + b->goff[inst];
    cudaMemcpyAsync(dst, host, sizeof(double) * (size_t)g.sx * g.sy, cudaMemcpyHostToDevice, b->st);
    return check("batch_upload");
} catch (...) {
    return asd2g::api_exception("asd2g_batch_upload");
}

int asd2g_batch_download(asd2g_batch *b, int inst, int field, double *host) try {
    const int slot = pad_slot(field);
    if (!b || !host || inst < 0 || inst >= b->count || slot < 0)
        return api_fail(ASD2G_E_ARG, "batch_download: bad instance or field (LS, KAPPA, H, DIV, PS, P)");
    const Grid &g = b->hinst[inst].g;
    const double *src = b->pad + (size_t)slot * b->gtot + b->goff[inst];
    cudaMemcpyAsync(host, src, sizeof(double) * (size_t)g.sx * g.sy, cudaMemcpyDeviceToHost, b->st);
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return check("batch_download");
    return check("batch_download");
} catch (...) {
    return asd2g::api_exception("asd2g_batch_download");
}

int asd2g_batch_field_ptr(asd2g_batch *b, int field, void **dptr, size_t *stride_doubles) try {
    const int slot = pad_slot(field);
    if (!b || !dptr || slot < 0) return api_fail(ASD2G_E_ARG, "batch_field_ptr: bad field");
    *dptr = b->pad + (size_t)slot * b->gtot;
    if (stride_doubles) *stride_doubles = b->gtot;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_field_ptr");
}

int asd2g_batch_offset(asd2g_batch *b, int inst, size_t *offset_doubles) try {
    if (!b || !offset_doubles || inst < 0 || inst >= b->count) return api_fail(ASD2G_E_ARG, "batch_offset: bad instance");
    *offset_doubles = b->goff[inst];
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_offset");
}

}  // extern "C"

namespace {
// dt[i] -> sc[0] of every instance (one strided copy).
int set_dts(asd2g_batch *b, const double *dt) {
    for (int i = 0; i < b->count; i++)
        if (!(dt[i] > 0.0) || !std::isfinite(dt[i])) return api_fail(ASD2G_E_ARG, "batch: dt must be positive and finite");
    cudaMemcpy2DAsync(b->sc, sizeof(double) * SC_PER_INST, dt, sizeof(double), sizeof(double), b->count,
                      cudaMemcpyHostToDevice, b->st);
    // the host array must outlive the copy
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return check("batch dt upload");
    return ASD2G_OK;
}

int solve_impl(asd2g_batch *b, double tol, int maxit, int *iters, double *rel_resid);
}  // namespace

extern "C" {

int asd2g_batch_assemble(asd2g_batch *b, const double *dt) try {
    NvtxRange nv("batched GFM assembly");
    if (!b || !dt) return api_fail(ASD2G_E_ARG, "batch_assemble: null argument");
    int rc = set_dts(b, dt);
    if (rc) return rc;
    launch_batch_assemble(b->dinst, b->cell_tiles, b->ncell_tiles, b->st);
    return check("batch_assemble");
} catch (...) {
    return asd2g::api_exception("asd2g_batch_assemble");
}

int asd2g_batch_solve(asd2g_batch *b, double tol, int maxit, int *iters, double *rel_resid) try {
    if (!b || !(tol > 0.0) || maxit < 1) return api_fail(ASD2G_E_ARG, "batch_solve: bad arguments");
    return solve_impl(b, tol, maxit, iters, rel_resid);
} catch (...) {
    return asd2g::api_exception("asd2g_batch_solve");
}

// The full droplet step of every instance (asd2g_droplet_step per instance,
// MG-FCG pressure solve), one launch per phase for the whole batch.
int asd2g_batch_step(asd2g_batch *b, double *dt, int reinit_mode, double tol, int maxit, int *iters,
                     double *rel_resid) try {
    NvtxRange nv("asd2g_batch_step");
    if (!b || !dt || !(tol > 0.0) || maxit < 1) return api_fail(ASD2G_E_ARG, "batch_step: bad arguments");
    if (reinit_mode < ASD2G_REINIT_ORIGINAL || reinit_mode > ASD2G_REINIT_MINRK2_SUSSMAN ||
        reinit_mode == ASD2G_REINIT_FIRSTTIME)
        return api_fail(ASD2G_E_UNSUPPORTED, "batch_step implements reinit modes 0, 1, 2 and 4");
    const bool sussman = reinit_mode == ASD2G_REINIT_SUSSMAN || reinit_mode == ASD2G_REINIT_MINRK2_SUSSMAN;
    if (sussman && b->splan.any_mixed)
        return api_fail(ASD2G_E_UNSUPPORTED, "batch_step: mixed-precision instances implement reinit modes 0 and 2");
    // instances keep their own time order and reinitialisation step count:
    // the phases run up to the largest, instances without a phase skip it
    int steps = 0, omax = 0;
    for (int i = 0; i < b->count; i++) {
        const asd2g_params &pp = b->prm[i];
        if (pp.precision != ASD2G_PRECISION_FP64 && pp.precision != ASD2G_PRECISION_MIXED)
            return api_fail(ASD2G_E_UNSUPPORTED, "batch_step runs FP64 and mixed-precision instances");
        if (pp.time_order < 0 || pp.time_order > 2)
            return api_fail(ASD2G_E_UNSUPPORTED, "batch_step implements time orders 0, 1 and 2");
        steps = b->hinst[i].nreinit > steps ? b->hinst[i].nreinit : steps;
        omax = pp.time_order > omax ? pp.time_order : omax;
    }
    int rc = set_dts(b, dt);
    if (rc) return rc;
    const BStepPlan &P = b->splan;
    cudaStream_t st = b->st;
    const size_t slot_bytes = sizeof(double) * b->gtot;
    auto slot = [&](int f) { return b->pad + (size_t)f * b->gtot; };
    // Solve_LevelSet_2D: lsB = ls; centred velocities; TVD-RK3 of HJ-WENO5
    cudaMemcpyAsync(slot(BS_LSB), slot(BS_LS), slot_bytes, cudaMemcpyDeviceToDevice, st);
    launch_bstep_center_vel(P, st);
    launch_bstep_fill_p(P, BS_LS, false, st);
    launch_bstep_ls_stage(P, 1, BS_LS, BS_LS, BS_W1, st);
    launch_bstep_ls_stage(P, 2, BS_W1, BS_LS, BS_W2, st);
    launch_bstep_ls_stage(P, 3, BS_W2, BS_LS, BS_LS, st);
    // reinitialisation (levelset2d.cpp:264-316, :433-486): lsInit, then the pseudo-steps
    if (reinit_mode == ASD2G_REINIT_MINRK2 || reinit_mode == ASD2G_REINIT_MINRK2_SUSSMAN) {
        launch_bstep_fill_p(P, BS_LS, false, st);
        cudaMemcpyAsync(slot(BS_LS0), slot(BS_LS), slot_bytes, cudaMemcpyDeviceToDevice, st);
    } else {
        cudaMemcpyAsync(slot(BS_LS0), slot(BS_LS), slot_bytes, cudaMemcpyDeviceToDevice, st);
        launch_bstep_fill_p(P, BS_LS, false, st);
    }
    // the Sussman modes start from zeroed work arrays (levelset2d.cpp:329-331;
    // their ghosts and corners stay 0): W1 (Sussman), W2 (both)
    if (reinit_mode == ASD2G_REINIT_SUSSMAN) cudaMemsetAsync(slot(BS_W1), 0, slot_bytes, st);
    if (sussman) cudaMemsetAsync(slot(BS_W2), 0, slot_bytes, st);
    for (int k = 0; k < steps; k++) {
        launch_bstep_reinit_pass(P, reinit_mode, 0, k, st);
        launch_bstep_reinit_pass(P, reinit_mode, 1, k, st);
        if (sussman) launch_bstep_reinit_pass(P, reinit_mode, 2, k, st);
    }
    // mixed instances: the same level-set step in FP32 (a session's
    // launch_ls_step32: LS with its ghosts -> FP32, centred velocities, three
    // packed WENO5/TVD-RK3 stages, lsInit, the packed reinitialisation
    // pseudo-steps, FP32 -> LS with its ghosts); the FP64 kernels above
    // skipped these instances and only refilled their P ghosts
    if (P.any_mixed) {
        launch_bstep_ls32_convert(P, false, st);
        launch_bstep_center_vel32(P, st);
        launch_bstep_ls_stage32(P, 1, 0, 0, 2, st);  // phi -> a
        launch_bstep_ls_stage32(P, 2, 2, 0, 3, st);  // a -> b
        launch_bstep_ls_stage32(P, 3, 3, 0, 0, st);  // b -> phi
        // lsInit: the phi array of the FP32 arena -> its ls0 array, every mixed
        // instance at once (the first mixed instance starts both arrays)
        int first = 0;
        while (!b->hinst[first].mixed) first++;
        const Ls32Work &w0 = b->hinst[first].w32;
        cudaMemcpyAsync(w0.ls0, w0.phi, sizeof(float) * (size_t)(w0.ls0 - w0.phi), cudaMemcpyDeviceToDevice, st);
        for (int k = 0; k < steps; k++) {
            launch_bstep_reinit32(P, reinit_mode, false, k, st);
            launch_bstep_reinit32(P, reinit_mode, true, k, st);
        }
        launch_bstep_ls32_convert(P, true, st);
    }
    // curvature (with the ghost fill of SolvePoisson's recompute), Heaviside, volume check
    launch_bstep_kappa(P, st);
    launch_bstep_fill_p(P, BS_KAPPA, true, st);
    launch_bstep_heaviside(P, st);
    launch_bstep_volume(P, st);
    // intermediate velocity (GetIntermediateVel, smoothed Heaviside), its divergence
    launch_bstep_mom_slot(P, 0, st);
    if (omax >= 1) {
        launch_bstep_fill_uv(P, BS_UA, BS_VA, st, 1);
        launch_bstep_mom_slot(P, 1, st);
    }
    if (omax >= 2) {
        launch_bstep_fill_uv(P, BS_UB, BS_VB, st, 2);
        launch_bstep_mom_slot(P, 2, st);
    }
    launch_bstep_fill_uv(P, BS_UHAT, BS_VHAT, st);
    cudaMemsetAsync(slot(BS_DIV), 0, slot_bytes, st);
    launch_bstep_divergence(P, st);
    // GFM assembly and the batched MG-FCG
    launch_batch_assemble(b->dinst, b->cell_tiles, b->ncell_tiles, st);
    rc = check("batch_step (before the solve)");
    if (rc) return rc;
    const int st_solve = solve_impl(b, tol, maxit, iters, rel_resid);
    if (st_solve < 0) return st_solve;
    // projection and the next dt
    launch_bstep_update_vel(P, st);
    launch_bstep_update_dt(P, st);
    cudaMemcpy2DAsync(dt, sizeof(double), b->sc + 1, sizeof(double) * SC_PER_INST, sizeof(double), b->count,
                      cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check("batch_step");
    rc = check("batch_step");
    return rc ? rc : st_solve;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_step");
}

int asd2g_batch_volume(asd2g_batch *b, double *sharp, double *smooth) try {
    if (!b) return api_fail(ASD2G_E_ARG, "null batch");
    if (sharp)
        cudaMemcpy2DAsync(sharp, sizeof(double), b->sc + 2, sizeof(double) * SC_PER_INST, sizeof(double), b->count,
                          cudaMemcpyDeviceToHost, b->st);
    if (smooth)
        cudaMemcpy2DAsync(smooth, sizeof(double), b->sc + 3, sizeof(double) * SC_PER_INST, sizeof(double), b->count,
                          cudaMemcpyDeviceToHost, b->st);
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return check("batch_volume");
    return check("batch_volume");
} catch (...) {
    return asd2g::api_exception("asd2g_batch_volume");
}

}  // extern "C"

namespace {
// Tile-shape tuning on this batch's own hierarchy (first solve only, after
// the multigrid set-up): four FCG iterations per shape, none allowed to stop
// early.  Leaves the fastest shape selected; the caller sets the solver
// scalars again.
int tune_shape(asd2g_batch *b) {
    if (b->shape_tuned || b->shape_forced >= 0) return ASD2G_OK;
    const BatchPlan &P = b->plan;
    struct Events {  // destroyed on every exit path
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } ev;
    if (cudaEventCreate(&ev.e0) != cudaSuccess || cudaEventCreate(&ev.e1) != cudaSuccess)
        return check("batch tile tuning events");
    cudaEvent_t e0 = ev.e0, e1 = ev.e1;
    int best = 0;
    for (int sh = 0; sh < MG_NSHAPES; sh++) {
        int rc = set_mg_shape(b, sh);
        if (rc) return rc;
        launch_batch_set_kstate(P, 0.0, 1 << 30, b->st);
        launch_batch_fcg_init(P, b->st);
        launch_batch_fcg_iter(P, 0, b->st);  // first launch of this shape's kernels
        cudaEventRecord(e0, b->st);
        for (int k = 0; k < 4; k++) launch_batch_fcg_iter(P, (k + 1) & 1, b->st);
        cudaEventRecord(e1, b->st);
        if (cudaEventSynchronize(e1) != cudaSuccess) return check("batch tile tuning");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        b->shape_ms[sh] = ms;
        if (ms < b->shape_ms[best]) best = sh;
    }
    b->shape_tuned = true;
    int rc = set_mg_shape(b, best);
    if (rc) return rc;
    return ASD2G_OK;
}

int solve_impl(asd2g_batch *b, double tol, int maxit, int *iters, double *rel_resid) {
    NvtxRange nv("batched pressure solve");
    const BatchPlan &P = b->plan;
    launch_batch_set_kstate(P, tol, maxit, b->st);
    launch_batch_mg_setup(P, b->st);
    int rc = tune_shape(b);
    if (rc) return rc;
    launch_batch_set_kstate(P, tol, maxit, b->st);
    launch_batch_fcg_init(P, b->st);
    rc = check("batch solve set-up");
    if (rc) return rc;
    if (!b->chunk_exec) {
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return check("capture");
        for (int k = 0; k < FCG_CHUNK_ITERS; k++) launch_batch_fcg_iter(P, k & 1, b->st);
        launch_batch_fcg_check(P, b->st);
        if (cudaStreamEndCapture(b->st, &graph) != cudaSuccess) return check("capture end");
        const cudaError_t e = cudaGraphInstantiate(&b->chunk_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return check("graph instantiate");
    }
    bool all_done = false;
    for (int launched = 0; !all_done && launched < maxit + 2 * FCG_CHUNK_ITERS; launched += FCG_CHUNK_ITERS) {
        if (cudaGraphLaunch(b->chunk_exec, b->st) != cudaSuccess) return check("graph launch");
        cudaMemcpyAsync(b->ks_host, b->ks, sizeof(KState) * b->count, cudaMemcpyDeviceToHost, b->st);
        if (cudaStreamSynchronize(b->st) != cudaSuccess) return check("batch solve");
        all_done = true;
        for (int i = 0; i < b->count; i++)
            if (!b->ks_host[i].done) all_done = false;
    }
    launch_batch_scatter(b->dinst, b->cell_tiles, b->ncell_tiles, b->st);
    rc = check("batch scatter");
    if (rc) return rc;
    int status = ASD2G_OK;
    for (int i = 0; i < b->count; i++) {
        const KState &k = b->ks_host[i];
        if (iters) iters[i] = k.it;
        if (rel_resid) rel_resid[i] = k.res;
        if (k.status == -5) status = api_fail(ASD2G_E_NONFINITE, "batch: non-finite residual");
        else if (k.status == -6) status = api_fail(ASD2G_E_BREAKDOWN, "batch: Krylov breakdown");
        else if (status == ASD2G_OK && !(!(k.res > tol) || k.status == 2)) status = ASD2G_NOT_CONVERGED;
    }
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return check("batch solve");
    return status;
}

// ------------------------------------------ learned preconditioner (UNET) --
constexpr int BPC_MAX_ITERS = 500;  // learned iterations before the MG-FCG fallback

// The network's correction on every every-th iteration of a chunk of
// FCG_CHUNK_ITERS (ASD2G_PC_EVERY = 1..8, default 8, as for single systems),
// besides the first application; the other iterations use the V-cycle alone.
bool pc_net_on(int k) {
    static const int every = [] {
        const char *e = std::getenv("ASD2G_PC_EVERY");
        const int v = e ? std::atoi(e) : 8;
        return v >= 1 && v <= 8 ? v : 8;
    }();
    return k % every == every - 1;
}

// Per-instance buffers of the learned preconditioner; instances with one grid
// size form a group whose feature and output planes are contiguous, so that
// one network pass serves the group.
int pc_alloc(asd2g_batch *b) {
    if (b->pc_ready) return ASD2G_OK;
    const int count = b->count;
    std::vector<int> gid(count);
    b->groups.clear();
    for (int i = 0; i < count; i++) {
        const Grid &g = b->hinst[i].g;
        int k = 0;
        while (k < (int)b->groups.size() && !(b->groups[k].nx == g.nx && b->groups[k].ny == g.ny)) k++;
        if (k == (int)b->groups.size()) b->groups.push_back({g.nx, g.ny, 0, nullptr, nullptr});
        gid[i] = k;
        b->groups[k].count++;
    }
    size_t ntot = 0;
    for (int i = 0; i < count; i++) ntot += (size_t)b->hinst[i].n;
    double *dv = nullptr;
    float *fv = nullptr;
    constexpr int NDV = 2 * FM_SLOTS + 1;  // direction slots p, q; r1
    int rc = balloc(b, &dv, NDV * ntot);
    if (!rc) rc = balloc(b, &fv, 5 * ntot + (size_t)count);  // features (4), output (1); scales
    if (rc) return rc;
    cudaMemsetAsync(dv, 0, sizeof(double) * NDV * ntot, b->st);
    cudaMemsetAsync(fv, 0, sizeof(float) * (5 * ntot + (size_t)count), b->st);
    // group planes in group order, instances in batch order inside a group
    std::vector<size_t> gbase(b->groups.size());
    size_t off = 0;
    for (size_t k = 0; k < b->groups.size(); k++) {
        gbase[k] = off;
        off += (size_t)b->groups[k].count * b->groups[k].nx * b->groups[k].ny;
        b->groups[k].feats = fv + 4 * gbase[k];
        b->groups[k].out = fv + 4 * ntot + gbase[k];
    }
    std::vector<size_t> gused(b->groups.size(), 0);
    size_t voff = 0;
    for (int i = 0; i < count; i++) {
        BInst &I = b->hinst[i];
        const int k = gid[i];
        const size_t at = gbase[k] + gused[k];
        gused[k] += (size_t)I.n;
        I.pc_feats = fv + 4 * at;
        I.pc_out = fv + 4 * ntot + at;
        I.pc_scal = fv + 5 * ntot + i;
        for (int j = 0; j < FM_SLOTS; j++) {
            I.fm.p[j] = dv + (size_t)j * ntot + voff;
            I.fm.q[j] = dv + (size_t)(FM_SLOTS + j) * ntot + voff;
        }
        I.pc_r1 = dv + (size_t)2 * FM_SLOTS * ntot + voff;
        voff += (size_t)I.n;
    }
    cudaMemcpyAsync(b->dinst, b->hinst.data(), sizeof(BInst) * count, cudaMemcpyHostToDevice, b->st);
    b->pc_ready = true;
    return check("learned preconditioner buffers");
}

// z = V-cycle(r) [+ omega u with u = network(r - A z)] for every instance
int pc_correct(asd2g_batch *b, bool with_net) {
    const BatchPlan &P = b->plan;
    if (with_net) {
        launch_batch_pc_input(P, b->st);
        for (const auto &G : b->groups) {
            const int rc = asd2g_unet_forward(b->net, G.count, G.nx, G.ny, G.feats, G.out);
            if (rc) return rc;
        }
    }
    launch_batch_pc_output(P, with_net, b->st);
    return check("batched learned preconditioner");
}

// FCG_CHUNK_ITERS truncated-FCG iterations (direction slot k % FM_SLOTS), the
// FP64 residual check, and the V-cycle alone after a restart
int pc_chunk(asd2g_batch *b) {
    const BatchPlan &P = b->plan;
    for (int k = 0; k < FCG_CHUNK_ITERS; k++) {
        launch_batch_pcm_iter(P, k % FM_SLOTS, b->st);
        const int rc = pc_correct(b, pc_net_on(k));
        if (rc) return rc;
    }
    launch_batch_fcg_check(P, b->st);
    return pc_correct(b, false);
}
static_assert(FCG_CHUNK_ITERS % FM_SLOTS == 0, "every replay of a chunk must write the direction slots in the same order");

int solve_learned_impl(asd2g_batch *b, double tol, int maxit, int *iters, double *rel_resid) {
    NvtxRange nv("batched pressure solve (learned preconditioner)");
    if (!b->net) return api_fail(ASD2G_E_ARG, "no preconditioner network attached (asd2g_batch_set_preconditioner_net)");
    const BatchPlan &P = b->plan;
    const int cap = maxit < BPC_MAX_ITERS ? maxit : BPC_MAX_ITERS;
    b->last_fallback = 0;
    launch_batch_set_kstate(P, tol, cap, b->st, ASD2G_SOLVER_UNET);
    launch_batch_mg_setup(P, b->st);
    int rc = tune_shape(b);
    if (rc) return rc;
    launch_batch_set_kstate(P, tol, cap, b->st, ASD2G_SOLVER_UNET);
    launch_batch_pc_setup(P, b->st);
    launch_batch_fcg_init(P, b->st);  // r = b, x = 0, z = V-cycle(r)
    rc = pc_correct(b, true);
    if (rc) return rc;
    if (!b->pc_exec) {
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return check("capture");
        const int rc2 = pc_chunk(b);
        if (cudaStreamEndCapture(b->st, &graph) != cudaSuccess) return check("capture end");
        if (rc2) {
            cudaGraphDestroy(graph);
            return rc2;
        }
        const cudaError_t e = cudaGraphInstantiate(&b->pc_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return check("graph instantiate");
    }
    bool all_done = false;
    for (int launched = 0; !all_done && launched < cap + 2 * FCG_CHUNK_ITERS; launched += FCG_CHUNK_ITERS) {
        if (cudaGraphLaunch(b->pc_exec, b->st) != cudaSuccess) return check("graph launch");
        cudaMemcpyAsync(b->ks_host, b->ks, sizeof(KState) * b->count, cudaMemcpyDeviceToHost, b->st);
        if (cudaStreamSynchronize(b->st) != cudaSuccess) return check("batch solve");
        all_done = true;
        for (int i = 0; i < b->count; i++)
            if (!b->ks_host[i].done) all_done = false;
    }
    int net_flag = 0;
    asd2g_unet_error_flag(b->net, &net_flag);
    bool ok = all_done && !net_flag;
    for (int i = 0; i < b->count && ok; i++) {
        const KState &k = b->ks_host[i];
        ok = (k.status == 0 || k.status == 2) && (!(k.res > tol) || k.status == 2);
    }
    if (!ok) {
        // the batched MG-FCG from zero, judged by the same FP64 residual
        std::vector<int> it1(b->count);
        for (int i = 0; i < b->count; i++) it1[i] = b->ks_host[i].it;
        b->last_fallback = 1;
        const int st2 = solve_impl(b, tol, maxit, iters, rel_resid);
        if (iters)
            for (int i = 0; i < b->count; i++) iters[i] += it1[i];
        return st2;
    }
    launch_batch_scatter(b->dinst, b->cell_tiles, b->ncell_tiles, b->st);
    rc = check("batch scatter");
    if (rc) return rc;
    for (int i = 0; i < b->count; i++) {
        if (iters) iters[i] = b->ks_host[i].it;
        if (rel_resid) rel_resid[i] = b->ks_host[i].res;
    }
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return check("batch solve");
    return ASD2G_OK;
}

}  // namespace

extern "C" {

int asd2g_batch_tile_shape(asd2g_batch *b, int *rows, int *cols, float *trial_ms) try {
    if (!b) return api_fail(ASD2G_E_ARG, "null batch");
    if (rows) *rows = MG_SHAPES[b->plan.shape][0];
    if (cols) *cols = MG_SHAPES[b->plan.shape][1];
    if (trial_ms)
        for (int k = 0; k < MG_NSHAPES; k++) trial_ms[k] = (float)b->shape_ms[k];
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_tile_shape");
}

int asd2g_batch_set_preconditioner_net(asd2g_batch *b, asd2g_unet *net) try {
    if (!b) return api_fail(ASD2G_E_ARG, "null batch");
    if (b->pc_exec) {  // the captured chunk holds the previous network's launches
        cudaGraphExecDestroy(b->pc_exec);
        b->pc_exec = nullptr;
    }
    if (!net) return ASD2G_OK;
    for (int i = 0; i < b->count; i++)
        if (b->hinst[i].g.nx % 8 || b->hinst[i].g.ny % 8)
            return api_fail(ASD2G_E_UNSUPPORTED, "the learned preconditioner needs nx and ny multiples of 8");
    int rc = pc_alloc(b);
    if (rc) return rc;
    if (!b->net) {
        // the batch's own network, its activation buffers sized for the largest size group
        size_t maxpix = 0;
        for (const auto &G : b->groups) {
            const size_t px = (size_t)G.count * G.nx * G.ny;
            maxpix = px > maxpix ? px : maxpix;
        }
        const size_t w = (maxpix / 8 + 7) / 8 * 8;
        if (w > (size_t)1 << 30) return api_fail(ASD2G_E_UNSUPPORTED, "batch too large for one network pass");
        rc = asd2g_unet_create(1, 8, (int)w, b->st, &b->net);
        if (rc) return rc;
    }
    std::vector<float> h(asd2g_unet_nparams(net));
    if (h.size() != asd2g_unet_nparams(b->net)) return api_fail(ASD2G_E_ARG, "network size mismatch");
    rc = asd2g_unet_get_params(net, h.data());
    if (!rc) rc = asd2g_unet_set_params(b->net, h.data());
    return rc;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_set_preconditioner_net");
}

int asd2g_batch_solve_with(asd2g_batch *b, int solver, double tol, int maxit, int *iters, double *rel_resid) try {
    if (!b || !(tol > 0.0) || maxit < 1) return api_fail(ASD2G_E_ARG, "batch_solve: bad arguments");
    if (solver == ASD2G_SOLVER_MGPCG) return solve_impl(b, tol, maxit, iters, rel_resid);
    if (solver == ASD2G_SOLVER_UNET) return solve_learned_impl(b, tol, maxit, iters, rel_resid);
    return api_fail(ASD2G_E_ARG, "batch solver must be ASD2G_SOLVER_MGPCG or ASD2G_SOLVER_UNET");
} catch (...) {
    return asd2g::api_exception("asd2g_batch_solve_with");
}

int asd2g_batch_last_fallback(asd2g_batch *b, int *used) try {
    if (!b || !used) return api_fail(ASD2G_E_ARG, "null argument");
    *used = b->last_fallback;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_last_fallback");
}

int asd2g_batch_sync(asd2g_batch *b) try {
    if (!b) return api_fail(ASD2G_E_ARG, "null batch");
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return check("batch sync");
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_batch_sync");
}

}  // extern "C"
