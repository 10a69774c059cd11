// Host side of libddagpu: contexts, the DDA_FFT driver over the device kernels, the
// batched orientation solves and the C ABI of include/ddagpu.h.
//
// The solver driver mirrors DDA_FFT (dda_func.cpp:1075-1570) step by step: step 0, the
// per-method recurrences, the absolute Error_max test and the best-iterate rollback.  All
// fields, reductions and coefficients stay on the device; the host only launches kernels
// and reads one flag per right-hand side per iteration to stop when all have converged.
#include <cuda.h>   // CUtensorMap and cuTensorMapEncodeTiled's types (the function comes
                    // from the runtime's driver entry point, no link to libcuda)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ddagpu.h"
#include "targets.h"
#include "internal.h"
#include "post.h"
#include "solver.h"
#include "fp64.h"

using namespace ddagpu;

namespace {
thread_local std::string g_err;
}

namespace ddagpu {
// the message behind ddagpu_last_error for the calling thread (also used by state.cpp)
int set_error(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}
}  // namespace ddagpu

namespace {

int fail(int code, const std::string &msg) { return set_error(code, msg); }

#define CK(expr)                                                                            \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess)                                                              \
            return fail(_e == cudaErrorMemoryAllocation ? DDAGPU_ENOMEM : DDAGPU_ECUDA,     \
                        std::string(#expr) + ": " + cudaGetErrorString(_e));                \
    } while (0)

#define RET(expr)                                                                           \
    do {                                                                                    \
        int _r = (expr);                                                                    \
        if (_r != DDAGPU_OK) return _r;                                                     \
    } while (0)

bool pow2_in(int n) { return n >= kMinEdge && n <= kMaxEdge && (n & (n - 1)) == 0; }

template <class T>
cudaError_t dalloc(T **p, size_t n)
{
    return cudaMalloc((void **)p, (n ? n : 1) * sizeof(T));
}

}  // namespace

struct ddagpu_ctx {
    int dev = 0;
    int ni = 0, nj = 0, nl = 0;
    size_t N = 0;
    double kd = 0;
    int cap = 0;
    cudaStream_t st = nullptr;
    Lat L{};
    int tile_x = 32, rows_g = 16;
    int fast = 0;                // compile-time-sized passes in use
    int fx = 0, fyz = 0;         // their launch variants (x pass, y/z passes)
    float2 *ahat = nullptr, *tw = nullptr;
    float2 *work = nullptr, *p = nullptr, *pmin = nullptr, *r = nullptr, *s = nullptr,
           *g = nullptr, *h = nullptr, *w = nullptr;
    RhsState *state = nullptr;
    int *active = nullptr;
    double *trace = nullptr;
    int trace_len = 0;
    signed char *occ = nullptr;
    int *mv = nullptr;
    float2 *alpha = nullptr;
    int nmat_cap = kMaxMaterials + 1;
    double *kinc = nullptr, *einc = nullptr;
    float2 *inc_tab = nullptr;   // [max_rhs][nj + nl + ni] incident phase tables
    // pinned host staging of the batched calls' inputs and outputs, grown on demand (the
    // copies from and to it are asynchronous, unlike those of pageable memory)
    unsigned char *pin = nullptr;
    size_t pin_bytes = 0;
    // post-processing buffers, grown on demand
    int ndir_cap = 0;
    double *ksc = nullptr, *esc_acc = nullptr, *cc_acc = nullptr, *normals = nullptr,
           *mueller = nullptr;
    float2 *esc = nullptr;
    float *cabs = nullptr, *cext = nullptr;
    int nplane_cap = 0, nangle_cap = 0;
    float2 *b32 = nullptr, *rb = nullptr;   // refinement: outer and inner right-hand sides
    double2 *x64 = nullptr;                 // refinement: FP64 solution
    bool occ_valid = false;      // occupancy of the last batched call is resident
    std::vector<signed char> occ_host;   // host copy of the occupancy in c->occ (if cached)
    std::vector<int> mv_host;            // and the material flags it was counted with
    int occ_host_nact = 0;
    signed char *occ_b = nullptr;   // [cap][N] per-right-hand-side occupancy (realisations)
    int *ndip = nullptr;            // [cap] dipoles of each rasterised realisation
    size_t occ_stride = 0;          // N while occ_b is in use, 0 otherwise
    int occ_nmat1 = 0, occ_nact = 0;
    long long launches = 0;      // kernels launched by this context
    // solver iterations 2.. as one CUDA graph: a conditional while node whose body is one
    // iteration, its step counter on the device (kept per context, rebuilt when the solve's
    // shape changes)
    int graph_on = 1;
    int *step_dev = nullptr;
    struct GraphKey {
        int solver, nrhs, max_step, nmat1, fast, fx, fyz, tile_x, rows_g, tlen, pair;
        float tau, err_max;
        double d0;
        size_t occ_stride;
        const void *trace, *occ;
        long long post, kz;
    } gkey{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    GraphKey wkey{};                 // the whole-solve graph of batched calls
    cudaGraph_t wgraph = nullptr;
    cudaGraphExec_t wexec = nullptr;
    long long w_fixed = 0, w_per_iter = 0;
    int w_matvec0 = 0, w_matvec_it = 0;
    int *nact_dev = nullptr;         // [cap] active cells per right-hand side
    int *err_dev = nullptr;          // set by a kernel whose bounded wait gave up
    void *worm_buf = nullptr;        // monomers of the realisation being rasterised
    size_t worm_bytes = 0;
    int wait_selftest = 0;           // 1: the x pass's wait waits for a phase nothing completes
    long long post_key = 0;          // shape of the post-processing recorded with a solve
    // far field by kz groups: the plan of the directions last uploaded, its device tables
    ddagpu::KzPlan kz;
    int ff_mode = 0;                 // ddagpu_set_farfield_mode
    int *kz_tab = nullptr;
    double *kz_val = nullptr;
    float2 *kz_sum = nullptr;
    size_t kz_tab_cap = 0, kz_val_cap = 0, kz_sum_cap = 0;
    // TMA tensor maps of the work buffer, one per x-pass column tile (x variants 9..11)
    alignas(64) CUtensorMap tmaps[3];
    bool has_tmap = false;
    Fp64Buffers *f64 = nullptr;  // FP64 solve buffers (ddagpu_solve_fp64), built on first use
    MixedCgBuffers *mcg = nullptr;   // FP64 fields of the mixed-precision CG refinement
    long long gen = 0;           // bumped whenever recorded graphs must be dropped
    int pair_step0 = 0;          // step 0 of a batched call: polarisation pairs share phi
    long long g_per_iter = 0;    // kernels in one recorded iteration
    long long graph_runs = 0;    // graph launches by this context
    std::mutex mu;
};

namespace {

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// The work buffer [cap][3][ni][2nj][2nl] complex float as a 5-D tensor map per x-pass
// column tile (box TL x 1 x ni x 1 x 1, 8-byte elements, no swizzle, no multicast), for the
// TMA variants of the x pass.  false if the driver does not offer the encoder.
bool encode_work_maps(ddagpu_ctx *c)
{
    typedef CUresult (*Encode)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                               const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                               CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                               CUtensorMapFloatOOBfill);
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
        return false;
    const Encode encode = reinterpret_cast<Encode>(fn);
    const cuuint64_t e = sizeof(float2);
    const cuuint64_t dim[5] = {(cuuint64_t)2 * c->nl, (cuuint64_t)2 * c->nj, (cuuint64_t)c->ni, 3,
                               (cuuint64_t)c->cap};
    const cuuint64_t str[4] = {dim[0] * e, dim[0] * dim[1] * e, dim[0] * dim[1] * dim[2] * e,
                               dim[0] * dim[1] * dim[2] * 3 * e};
    const cuuint32_t one[5] = {1, 1, 1, 1, 1};
    for (int v = 0; v < 3; v++) {
        const int tl = matvec_fast_x_tile(c->ni, v);
        if (tl < 2 || (tl * e) % 16 != 0) return false;
        const cuuint32_t box[5] = {(cuuint32_t)tl, 1, (cuuint32_t)c->ni, 1, 1};
        if (encode(&c->tmaps[v], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, c->work, dim, str, box, one,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

// W_n^k (k < n) followed by W_2n^j (j < n), forward sign, built in FP64.
void twiddles(int n, float2 *out)
{
    const double pi = 3.14159265358979323846264338327950288;
    for (int k = 0; k < n; k++)
        out[k] = make_float2((float)std::cos(-2.0 * pi * k / n), (float)std::sin(-2.0 * pi * k / n));
    for (int j = 0; j < n; j++)
        out[n + j] = make_float2((float)std::cos(-pi * j / n), (float)std::sin(-pi * j / n));
}

// A kernel of the context gave up a bounded wait (its bulk copies did not complete):
// report it and clear the flag for the next call.
int device_wait_error(ddagpu_ctx *c, int flag)
{
    if (!flag) return DDAGPU_OK;
    cudaMemsetAsync(c->err_dev, 0, sizeof(int), c->st);
    cudaStreamSynchronize(c->st);
    return fail(DDAGPU_ECUDA, "a device wait ran out (asynchronous copy not completed)");
}

// Forget the recorded solve graphs (they hold buffer addresses about to change).
void drop_graphs(ddagpu_ctx *c)
{
    c->gen += 1;   // a group's graph holding this context is rebuilt too
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->wexec) cudaGraphExecDestroy(c->wexec);
    if (c->wgraph) cudaGraphDestroy(c->wgraph);
    c->gexec = nullptr;
    c->graph = nullptr;
    c->wexec = nullptr;
    c->wgraph = nullptr;
}

int ensure_post(ddagpu_ctx *c, int ndir, int nplanes, int nangles)
{
    if (ndir > c->ndir_cap || nplanes > c->nplane_cap || nangles > c->nangle_cap) drop_graphs(c);
    if (ndir > c->ndir_cap) {
        cudaFree(c->ksc);
        cudaFree(c->esc_acc);
        cudaFree(c->esc);
        c->ksc = nullptr;
        c->esc_acc = nullptr;
        c->esc = nullptr;
        CK(dalloc(&c->ksc, (size_t)c->cap * ndir * 3));
        CK(dalloc(&c->esc_acc, (size_t)c->cap * ndir * 6));
        CK(dalloc(&c->esc, (size_t)c->cap * ndir * 3));
        c->ndir_cap = ndir;
    }
    if (nplanes > c->nplane_cap || nangles > c->nangle_cap) {
        cudaFree(c->normals);
        cudaFree(c->mueller);
        c->normals = nullptr;
        c->mueller = nullptr;
        const int np = std::max(nplanes, c->nplane_cap), na = std::max(nangles, c->nangle_cap);
        CK(dalloc(&c->normals, (size_t)c->cap * np * 3));
        CK(dalloc(&c->mueller, (size_t)c->cap * na * 16));
        c->nplane_cap = np;
        c->nangle_cap = na;
    }
    return DDAGPU_OK;
}

MatvecArgs mv_args(ddagpu_ctx *c, int nrhs, const float2 *src, float2 *out, int epmode, float sv,
                   const float2 *v, int conj, int nmat1, bool gate)
{
    MatvecArgs a{};
    a.L = c->L;
    a.nrhs = nrhs;
    a.src = src;
    a.fstride = 3 * c->N;
    a.work = c->work;
    a.wstride = (size_t)3 * c->ni * (2 * c->nj) * (2 * c->nl);
    a.ahat = c->ahat;
    a.conj = conj;
    a.out = out;
    a.ep.mode = epmode;
    a.ep.conj = conj;
    a.ep.sv = sv;
    a.ep.v = v;
    a.ep.occ = c->occ_stride ? c->occ_b : c->occ;
    a.ep.occ_stride = c->occ_stride;
    a.ep.alpha = c->alpha;
    a.ep.mv = c->mv;
    a.ep.nmat1 = nmat1;
    a.rhs_active = gate ? c->active : nullptr;
    a.tile_x = c->tile_x;
    a.rows_g = c->rows_g;
    a.fast = c->fast;
    a.fx = c->fx;
    a.fyz = c->fyz;
    a.err = c->err_dev;
    a.wait_selftest = c->wait_selftest;
    a.tmaps = c->has_tmap ? (const void *)c->tmaps : nullptr;
    return a;
}

FieldArgs fa_args(ddagpu_ctx *c, int nrhs, int nmat1, double d0, float tau)
{
    FieldArgs f{};
    f.N = c->N;
    f.nrhs = nrhs;
    f.ni = c->ni;
    f.nj = c->nj;
    f.nl = c->nl;
    f.occ = c->occ_stride ? c->occ_b : c->occ;
    f.occ_stride = c->occ_stride;
    f.mv = c->mv;
    f.alpha = c->alpha;
    f.nmat1 = nmat1;
    f.st = c->state;
    f.rhs_active = c->active;
    f.p = c->p;
    f.pmin = c->pmin;
    f.r = c->r;
    f.s = c->s;
    f.g = c->g;
    f.h = c->h;
    f.w = c->w;
    f.kinc = c->kinc;
    f.einc = c->einc;
    f.d0 = d0;
    f.tau = tau;
    f.b = c->b32;
    f.rb = c->rb;
    f.x64 = c->x64;
    f.rhs_in = nullptr;
    return f;
}

struct SolveResult {
    std::vector<RhsState> st;
    std::vector<double> trace;
    int matvec0 = 0, matvec_it = 0;
};

// The whole solve of a batch as graph nodes: step 0, the iterations as a conditional
// while node, the rollback and the post-processing.  Captured once per solve shape and
// kept in the context (or, for a group of contexts, in the group's graph, one independent
// branch per context); the inputs (fields, tables, occupancy, nact) are device buffers the
// host fills before each launch.
ddagpu_ctx::GraphKey whole_key(ddagpu_ctx *c, int nrhs, int solver, float tau, int max_step, float err_max,
                               int nmat1, double d0)
{
    ddagpu_ctx::GraphKey key{};
    key.solver = solver;
    key.nrhs = nrhs;
    key.max_step = max_step;
    key.nmat1 = nmat1;
    key.fast = c->fast;
    key.fx = c->fx;
    key.fyz = c->fyz;
    key.tile_x = c->tile_x;
    key.rows_g = c->rows_g;
    key.tlen = -1;                       // marks the whole-solve graph
    key.tau = tau;
    key.err_max = err_max;
    key.d0 = d0;
    key.occ_stride = c->occ_stride;
    key.trace = nullptr;
    key.occ = c->occ_stride ? (const void *)c->occ_b : (const void *)c->occ;
    key.post = c->post_key;
    key.kz = c->kz.groups ? ((long long)c->kz.groups << 32) | c->kz.items : 0;
    key.pair = c->pair_step0;
    return key;
}

// Records the whole solve into graph g as a branch with no dependencies; n_fixed and
// n_per_iter receive the kernels of the fixed part and of one loop pass.
template <class Step0, class Top, class Body>
int record_whole_solve(ddagpu_ctx *c, cudaGraph_t g, int nrhs, int max_step, float err_max, int nmat1,
                       double d0, float tau, Step0 &step0, Top &top, Body &body,
                       const std::function<int()> &post, long long &n_fixed, long long &n_per_iter)
{
    cudaStream_t st = c->st;
    const long long l_save = c->launches;
    auto give_up = [&](int rc, cudaError_t e, const char *what) {
        cudaStreamCaptureStatus cs;
        if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t t = nullptr;
            cudaStreamEndCapture(st, &t);
            if (t && t != g) cudaGraphDestroy(t);
        }
        c->launches = l_save;
        if (rc != DDAGPU_OK) return rc;
        return fail(DDAGPU_ECUDA, std::string("solve graph (") + what + "): " + cudaGetErrorString(e));
    };
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 0, 0);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "handle");
    const long long l0 = c->launches;
    // phase 1: fresh state, step 0, the convergence test of step 1, the loop condition
    e = cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "capture");
    int rc = DDAGPU_OK;
    e = launch_init_state(c->state, c->active, nrhs, (double)err_max, c->nact_dev, st);
    if (e == cudaSuccess) rc = step0();
    if (rc == DDAGPU_OK && e == cudaSuccess) e = launch_step_set(c->step_dev, 1, st);
    if (rc == DDAGPU_OK && e == cudaSuccess) rc = top(max_step, c->step_dev);
    if (rc == DDAGPU_OK && e == cudaSuccess)
        e = launch_loop_control(c->active, nrhs, c->step_dev, max_step, h, st);
    if (rc != DDAGPU_OK || e != cudaSuccess) return give_up(rc, e, "step 0");
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &ndeps);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "capture info");
    std::vector<cudaGraphNode_t> leaves(deps, deps + ndeps);
    cudaGraph_t t = nullptr;
    e = cudaStreamEndCapture(st, &t);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "end capture");
    const long long n_head = c->launches - l0 + 3;   // + init, step set, loop control
    // the while node and its body: one iteration, the next step's test, the condition
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t cn;
    e = cudaGraphAddNode(&cn, g, leaves.data(), leaves.size(), &np);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "while node");
    const long long l1 = c->launches;
    e = cudaStreamBeginCaptureToGraph(st, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "body capture");
    rc = body(max_step, c->step_dev, true);
    if (rc == DDAGPU_OK) e = launch_step_advance(c->step_dev, st);
    if (rc == DDAGPU_OK && e == cudaSuccess) rc = top(max_step, c->step_dev);
    if (rc == DDAGPU_OK && e == cudaSuccess)
        e = launch_loop_control(c->active, nrhs, c->step_dev, max_step, h, st);
    if (rc != DDAGPU_OK || e != cudaSuccess) return give_up(rc, e, "body");
    e = cudaStreamEndCapture(st, &t);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "end body capture");
    const long long n_body = c->launches - l1 + 2;
    // phase 3: rollback and post-processing after the loop
    const long long l2 = c->launches;
    e = cudaStreamBeginCaptureToGraph(st, g, &cn, nullptr, 1, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "tail capture");
    FieldArgs F = fa_args(c, nrhs, nmat1, d0, tau);
    e = launch_scalar(c->state, nullptr, nullptr, nrhs, SC_FINAL, 0, nullptr, 0, st);
    if (e == cudaSuccess) e = launch_gated_copy(F, 1, st);
    if (e == cudaSuccess) rc = post();
    if (rc != DDAGPU_OK || e != cudaSuccess) return give_up(rc, e, "tail");
    e = cudaStreamEndCapture(st, &t);
    if (e != cudaSuccess) return give_up(DDAGPU_OK, e, "end tail capture");
    const long long n_tail = c->launches - l2 + 2;
    n_fixed = n_head + n_tail;
    n_per_iter = n_body;
    c->launches = l_save;
    return DDAGPU_OK;
}

// Device results of a launched whole solve (on the context's stream): the solver states,
// the last step and the bounded-wait flag; counts the launched kernels.
int read_whole_solve(ddagpu_ctx *c, int nrhs, SolveResult &res, long long n_fixed, long long n_per_iter,
                     int matvec0, int matvec_it, bool own_launch = true)
{
    cudaStream_t st = c->st;
    int last = 1;
    res.st.resize((size_t)nrhs);
    CK(cudaMemcpyAsync(res.st.data(), c->state, nrhs * sizeof(RhsState), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last, c->step_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
    int werr = 0;
    CK(cudaMemcpyAsync(&werr, c->err_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    RET(device_wait_error(c, werr));
    c->launches += n_fixed + (long long)(last - 1) * n_per_iter;
    res.matvec0 = matvec0;
    res.matvec_it = matvec_it;
    if (own_launch) c->graph_runs += 1;   // a group's launch is counted by the group
    return DDAGPU_OK;
}

// A whole solve prepared for a group's graph instead of being launched (see ddagpu_group):
// the inputs are uploaded and the solve's graph key is returned; with graph set, the solve
// is also recorded into it as an independent branch.
struct GroupRecord {
    cudaGraph_t graph = nullptr;
    ddagpu_ctx::GraphKey key{};
    long long n_fixed = 0, n_per_iter = 0;
    int matvec0 = 0, matvec_it = 0;
};

template <class Step0, class Top, class Body>
int run_whole_graph(ddagpu_ctx *c, int nrhs, int solver, float tau, int max_step, float err_max,
                    int nmat1, double d0, int nact, const int *nact_per, SolveResult &res,
                    Step0 &step0, Top &top, Body &body, const std::function<int()> &post,
                    GroupRecord *rec)
{
    cudaStream_t st = c->st;
    std::vector<int> na((size_t)nrhs);
    for (int k = 0; k < nrhs; k++) na[(size_t)k] = nact_per ? nact_per[k] : nact;
    CK(cudaMemcpyAsync(c->nact_dev, na.data(), nrhs * sizeof(int), cudaMemcpyHostToDevice, st));
    const ddagpu_ctx::GraphKey key = whole_key(c, nrhs, solver, tau, max_step, err_max, nmat1, d0);
    if (rec) {   // for the group's graph; the group launches it and reads the results
        rec->key = key;
        if (!rec->graph) return DDAGPU_OK;
        RET(record_whole_solve(c, rec->graph, nrhs, max_step, err_max, nmat1, d0, tau, step0, top, body,
                               post, rec->n_fixed, rec->n_per_iter));
        rec->matvec0 = res.matvec0;
        rec->matvec_it = res.matvec_it;
        return DDAGPU_OK;
    }
    if (!c->wexec || std::memcmp(&key, &c->wkey, sizeof key) != 0) {
        if (c->wexec) cudaGraphExecDestroy(c->wexec);
        if (c->wgraph) cudaGraphDestroy(c->wgraph);
        c->wexec = nullptr;
        c->wgraph = nullptr;
        cudaGraph_t g = nullptr;
        CK(cudaGraphCreate(&g, 0));
        long long nf = 0, npi = 0;
        const int rc = record_whole_solve(c, g, nrhs, max_step, err_max, nmat1, d0, tau, step0, top, body,
                                          post, nf, npi);
        if (rc != DDAGPU_OK) {
            cudaGraphDestroy(g);
            return rc;
        }
        cudaGraphExec_t x = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&x, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return fail(DDAGPU_ECUDA, std::string("solve graph (instantiate): ") + cudaGetErrorString(e));
        }
        c->wgraph = g;
        c->wexec = x;
        c->wkey = key;
        c->w_fixed = nf;
        c->w_per_iter = npi;
        c->w_matvec0 = res.matvec0;
        c->w_matvec_it = res.matvec_it;
    }
    CK(cudaGraphLaunch(c->wexec, st));
    return read_whole_solve(c, nrhs, res, c->w_fixed, c->w_per_iter, c->w_matvec0, c->w_matvec_it);
}

// post (may be null): kernels issued after the solve on the context's stream (far field,
// cross sections, Mueller); with the solver graph on and no trace, step 0, the iterations,
// the rollback and post become one graph launch.
int run_solver(ddagpu_ctx *c, int nrhs, int solver, float tau, int max_step, float err_max,
               int nmat1, double d0, int nact, SolveResult &res, bool want_trace,
               const float2 *rhs_in = nullptr, const int *nact_per = nullptr,
               const std::function<int()> *post = nullptr, GroupRecord *rec = nullptr)
{
    if (solver < 0 || solver > 3) return fail(DDAGPU_EINVAL, "solver must be 0..3");
    if (max_step < 0) return fail(DDAGPU_EINVAL, "Max_Step must be >= 0");
    if (solver == 2 && (!c->g || !c->h)) return fail(DDAGPU_EINVAL, "no BiCGStab work space");
    cudaStream_t st = c->st;
    const int tl = max_step + 1;
    if (want_trace && tl > c->trace_len) {
        cudaFree(c->trace);
        c->trace = nullptr;
        CK(dalloc(&c->trace, (size_t)c->cap * tl));
        c->trace_len = tl;
    }
    double *trace = want_trace ? c->trace : nullptr;
    const int tlen = want_trace ? tl : 0;
    const bool whole = post && (c->graph_on || rec) && !want_trace && !rhs_in;
    if (rec && !whole) return fail(DDAGPU_EINVAL, "a group records whole batched solves only");
    if (!whole) {
        std::vector<RhsState> init((size_t)nrhs);
        for (int k = 0; k < nrhs; k++) {
            RhsState &S = init[(size_t)k];
            std::memset(&S, 0, sizeof S);
            S.err_max = (double)err_max;
            S.active = 1;
            S.nact = nact_per ? nact_per[k] : nact;
        }
        CK(cudaMemcpyAsync(c->state, init.data(), nrhs * sizeof(RhsState), cudaMemcpyHostToDevice, st));
        std::vector<int> ones((size_t)nrhs, 1);
        CK(cudaMemcpyAsync(c->active, ones.data(), nrhs * sizeof(int), cudaMemcpyHostToDevice, st));
    }

    FieldArgs F = fa_args(c, nrhs, nmat1, d0, tau);
    F.rhs_in = rhs_in;
    auto field = [&](int op) {
        c->launches += 1;
        return launch_field_op(op, F, st);
    };
    auto scal = [&](int stage, int step) {
        c->launches += 1;
        return launch_scalar(c->state, c->active, c->active, nrhs, stage, step, trace, tlen, st);
    };
    // out = sv v - alpha conv(src) on active cells, gated by the active flags
    auto matvec = [&](const float2 *src, float2 *out, float sv, const float2 *v, int conj) {
        c->launches += 3;
        return launch_matvec(mv_args(c, nrhs, src, out, 1, sv, v, conj, nmat1, true), st);
    };

    // ---- step 0 (dda_func.cpp:1102-1293): p = p_inc, or the given right-hand side
    auto step0 = [&]() -> int {
    if (!rhs_in && c->fast) {
        // the forward pass computes p_inc itself (from the phase tables) and stores it
        CK(launch_inc_tables(F, c->inc_tab, st));
        MatvecArgs m = mv_args(c, nrhs, c->p, c->r, 1, 0.f, nullptr, 0, nmat1, true);
        m.inc = 1;
        m.pair = (c->pair_step0 && nrhs % 2 == 0) ? 1 : 0;
        m.inc_tab = c->inc_tab;
        m.einc = c->einc;
        m.inc_out = c->p;
        c->launches += 4;
        CK(launch_matvec(m, st));   // p = p_inc, r = -alpha (G * p_inc)
    } else {
        if (rhs_in) CK(launch_refine(4, F, st));
        else CK(launch_first_approx(F, st));
        c->launches += 1;
        CK(matvec(c->p, c->r, 0.f, nullptr, 0));   // r = -alpha (G * p_inc)
    }
    res.matvec0 = 1;
    switch (solver) {
    case 0:   // s = r is deferred to the first iteration (an RHS converged at step 0 never needs it)
        CK(field(OP_ERR));
        CK(scal(SC_STEP0_ERR1, 0));
        break;
    case 1:
        CK(field(OP_STEP0_AA));
        CK(scal(SC_STEP0_AA, 0));
        CK(matvec(c->r, c->s, 1.f, c->r, 1));   // s = r - conj(alpha) conv*(r)
        res.matvec0 = 2;
        break;
    case 2:
        CK(field(OP_STEP0_BICG));
        CK(scal(SC_B_RHO1, 0));
        CK(matvec(c->s, c->h, 1.f, c->s, 0));
        CK(field(OP_B_GH));
        CK(scal(SC_B2, 0));
        CK(field(OP_B_R));
        CK(matvec(c->r, c->w, 1.f, c->r, 0));
        CK(field(OP_B_WW));
        CK(scal(SC_B3, 0));
        CK(field(OP_B_P));
        CK(scal(SC_B4, 0));
        res.matvec0 = 3;
        break;
    case 3:
        CK(field(OP_STEP0_SIMPLE));
        CK(scal(SC_STEP0_ERR1, 0));
        break;
    }
    CK(scal(SC_START, 0));
    // p_min = p (the step-0 iterate) is copied by the gated copy of the first iteration
    res.matvec_it = (solver == 1 || solver == 2) ? 2 : 1;
    return DDAGPU_OK;
    };

    // ---- iterations (dda_func.cpp:1301-1535)
    // top of an iteration: convergence test, best-iterate bookkeeping and copy
    auto top = [&](int o, const int *sdev) -> int {
        c->launches += 2;
        CK(launch_scalar(c->state, c->active, c->active, nrhs, SC_TOP, o, trace, tlen, st, sdev));
        CK(launch_gated_copy(F, 0, st));
        return DDAGPU_OK;
    };
    // the solver's recurrences of one iteration (gated per right-hand side by its flag);
    // gate_copy: CG's deferred s = r decided on the device (graph of the whole solve)
    auto body = [&](int o, const int *sdev, bool gate_copy = false) -> int {
        auto sc = [&](int stage) {
            c->launches += 1;
            return launch_scalar(c->state, c->active, c->active, nrhs, stage, o, trace, tlen, st, sdev);
        };
        switch (solver) {
        case 0:
            if (gate_copy) {
                FieldArgs G = F;
                G.step_gate = sdev;
                c->launches += 1;
                CK(launch_field_op(OP_COPY_RS, G, st));
            } else if (o == 1) {
                CK(field(OP_COPY_RS));
            }
            CK(matvec(c->s, c->w, 1.f, c->s, 0));
            CK(field(OP_CG1));
            CK(sc(SC_CG1));
            CK(field(OP_CG2));
            CK(sc(SC_CG2));
            CK(field(OP_CG3));
            break;
        case 1:
            CK(matvec(c->s, c->w, 1.f, c->s, 0));
            CK(field(OP_AA1));
            CK(sc(SC_AA1));
            CK(field(OP_AA2));
            CK(sc(SC_AA2));
            CK(matvec(c->r, c->w, 1.f, c->r, 1));
            CK(field(OP_AA3));
            break;
        case 2:
            CK(field(OP_B_RHO));
            CK(sc(SC_B1));
            CK(field(OP_B_S));
            CK(matvec(c->s, c->h, 1.f, c->s, 0));
            CK(field(OP_B_GH));
            CK(sc(SC_B2));
            CK(field(OP_B_R));
            CK(matvec(c->r, c->w, 1.f, c->r, 0));
            CK(field(OP_B_WW));
            CK(sc(SC_B3));
            CK(field(OP_B_P));
            CK(sc(SC_B4));
            break;
        case 3:
            CK(matvec(c->p, c->w, 1.f, c->p, 0));
            CK(field(OP_SIMPLE));
            CK(sc(SC_ERR1));
            break;
        }
        return DDAGPU_OK;
    };
    if (whole) return run_whole_graph(c, nrhs, solver, tau, max_step, err_max, nmat1, d0, nact,
                                      nact_per, res, step0, top, body, *post, rec);
    RET(step0());
    // iteration 1 (and all of them without the graph) from the host: the loop stops when
    // no right-hand side is left active (read back once per iteration)
    const bool use_graph = c->graph_on && max_step >= 2;
    std::vector<int> act((size_t)nrhs);
    bool graph_from_2 = false;
    for (int o = 1; o <= max_step; o++) {
        RET(top(o, nullptr));
        CK(cudaMemcpyAsync(act.data(), c->active, nrhs * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        bool any = false;
        for (int k = 0; k < nrhs; k++) any = any || act[(size_t)k];
        if (!any) break;
        if (use_graph && o == 2) {   // the top of step 2 ran; its body starts the graph
            graph_from_2 = true;
            break;
        }
        RET(body(o, nullptr));
    }
    if (graph_from_2) {
        // iterations 2..Max_Step: one graph launch; a pass of the while body is the
        // recurrences of one step, then the convergence test of the next step, and its
        // last kernel decides whether another pass follows
        ddagpu_ctx::GraphKey key{};
        key.solver = solver;
        key.nrhs = nrhs;
        key.max_step = max_step;
        key.nmat1 = nmat1;
        key.fast = c->fast;
        key.fx = c->fx;
        key.fyz = c->fyz;
        key.tile_x = c->tile_x;
        key.rows_g = c->rows_g;
        key.tlen = tlen;
        key.tau = tau;
        key.d0 = d0;
        key.occ_stride = c->occ_stride;
        key.trace = trace;
        key.occ = c->occ_stride ? (const void *)c->occ_b : (const void *)c->occ;
        if (!c->gexec || std::memcmp(&key, &c->gkey, sizeof key) != 0) {
            if (c->gexec) cudaGraphExecDestroy(c->gexec);
            if (c->graph) cudaGraphDestroy(c->graph);
            c->gexec = nullptr;
            c->graph = nullptr;
            cudaGraph_t g = nullptr;
            CK(cudaGraphCreate(&g, 0));
            cudaGraphConditionalHandle h;
            cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
            cudaGraphNodeParams np{};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            cudaGraphNode_t node;
            if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
            if (e == cudaSuccess)
                e = cudaStreamBeginCaptureToGraph(st, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) {
                cudaGraphDestroy(g);
                return fail(DDAGPU_ECUDA, std::string("solver graph: ") + cudaGetErrorString(e));
            }
            const long long l0 = c->launches;
            int rc = body(max_step, c->step_dev);
            cudaError_t le = rc == DDAGPU_OK ? launch_step_advance(c->step_dev, st) : cudaSuccess;
            if (rc == DDAGPU_OK && le == cudaSuccess) rc = top(max_step, c->step_dev);
            if (rc == DDAGPU_OK && le == cudaSuccess)
                le = launch_loop_control(c->active, nrhs, c->step_dev, max_step, h, st);
            cudaGraph_t captured = nullptr;
            const cudaError_t ee = cudaStreamEndCapture(st, &captured);
            c->g_per_iter = c->launches - l0 + 2;
            c->launches = l0;
            if (rc != DDAGPU_OK || le != cudaSuccess || ee != cudaSuccess) {
                cudaGraphDestroy(g);
                if (rc != DDAGPU_OK) return rc;
                return fail(DDAGPU_ECUDA, std::string("solver graph capture: ") +
                                              cudaGetErrorString(le != cudaSuccess ? le : ee));
            }
            cudaGraphExec_t x = nullptr;
            e = cudaGraphInstantiate(&x, g, 0);
            if (e != cudaSuccess) {
                cudaGraphDestroy(g);
                return fail(DDAGPU_ECUDA, std::string("solver graph instantiate: ") + cudaGetErrorString(e));
            }
            c->graph = g;
            c->gexec = x;
            c->gkey = key;
        }
        const int first = 2;
        CK(cudaMemcpyAsync(c->step_dev, &first, sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaGraphLaunch(c->gexec, st));
        int last = first;
        CK(cudaMemcpyAsync(&last, c->step_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        c->launches += (long long)(last - first) * c->g_per_iter;   // one pass per step advanced
        c->graph_runs += 1;
    }
    // ---- rollback (dda_func.cpp:1537-1548), for every right-hand side
    CK(launch_scalar(c->state, nullptr, nullptr, nrhs, SC_FINAL, 0, nullptr, 0, st));
    CK(launch_gated_copy(F, 1, st));
    c->launches += 2;
    if (post) RET((*post)());
    res.st.resize((size_t)nrhs);
    CK(cudaMemcpyAsync(res.st.data(), c->state, nrhs * sizeof(RhsState), cudaMemcpyDeviceToHost, st));
    if (want_trace) {
        res.trace.assign((size_t)nrhs * tl, 0.0);
        CK(cudaMemcpyAsync(res.trace.data(), c->trace, res.trace.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, st));
    }
    int werr = 0;
    CK(cudaMemcpyAsync(&werr, c->err_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    RET(device_wait_error(c, werr));
    return DDAGPU_OK;
}

int count_active(const signed char *occ, size_t N, const int *mv, int nmat1)
{
    int n = 0;
    for (size_t q = 0; q < N; q++) {
        const int m = (unsigned char)occ[q];
        if (m < nmat1 && mv[m]) n++;
    }
    return n;
}

int check_occ(const signed char *occ, size_t N, int nmat1)
{
    for (size_t q = 0; q < N; q++)
        if ((int)occ[q] < 0 || (int)occ[q] >= nmat1)
            return fail(DDAGPU_EINVAL, "cAlpha holds a material index outside 0..n_mat");
    return DDAGPU_OK;
}

// Polarisabilities (dda_func.cpp:1631-1677) in double.
struct cd {
    double r, i;
};
cd cmuld(cd a, cd b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
cd cdivd(cd a, cd b)
{
    const double d = b.r * b.r + b.i * b.i;
    return {(a.r * b.r + a.i * b.i) / d, (a.i * b.r - a.r * b.i) / d};
}
cd polarizability(int model, double d0, cd m, const double *kinc, const double *einc)
{
    const double pi = 3.14159265358979323846264338327950288;
    const cd eps = cmuld(m, m);
    cd a = cdivd({eps.r - 1.0, eps.i}, {eps.r + 2.0, eps.i});
    const double f = d0 * d0 * d0 * (0.75 / pi);
    a = {a.r * f, a.i * f};
    auto rr = [](cd x) { // x / (1 - (2/3) i x)
        return cdivd(x, {1.0 + (2.0 / 3.0) * x.i, -(2.0 / 3.0) * x.r});
    };
    if (model == 2) return rr(a);
    if (model == 3) {
        const double b = -std::sqrt(4.0 * pi / 3.0) / d0;
        return rr(cdivd(a, {1.0 + a.r * b, a.i * b}));
    }
    if (model == 4 || model == 5) {
        const double b1 = -1.8915316, b2 = 0.1648469, b3 = -1.7700004;
        double S = 0.2;
        if (model == 5) {
            const double rx = kinc[0] * einc[0], ry = kinc[1] * einc[2], rz = kinc[2] * einc[4];
            S = rx * rx + ry * ry + rz * rz;
        }
        const cd t = {b1 + b2 * eps.r + S * b3 * eps.r, b2 * eps.i + S * b3 * eps.i - (2.0 / 3.0) * d0};
        const cd ad = {a.r / d0, a.i / d0};
        const cd q = cmuld(ad, t);
        return cdivd(a, {1.0 + q.r, q.i});
    }
    return a;
}

int rounding_ref(float r0)
{ // complex.cpp:213-223
    double ip;
    const double fr = std::modf((double)r0, &ip);
    return fr > 0.5 ? (int)ip + 1 : (int)ip;
}

}  // namespace

extern "C" {

const char *ddagpu_version(void) { return "ddagpu 1.0 (sm_100a)"; }

int ddagpu_binary_version(int device, int *version)
{
    if (!version) return fail(DDAGPU_EINVAL, "null argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(DDAGPU_ENOTBUILT, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(DDAGPU_EINVAL, "bad device index");
    DevGuard dg(device);
    CK(kernel_binary_version(version));
    return DDAGPU_OK;
}
const char *ddagpu_last_error(void) { return g_err.c_str(); }

int ddagpu_num_angles(float theta_min, float theta_max, float theta_step)
{
    return rounding_ref(((theta_max - theta_min) / theta_step) + 1.f);
}

int ddagpu_create(ddagpu_ctx **out, int device, int i_max, int j_max, int l_max, double kd,
                  int max_rhs)
{
    if (!out) return fail(DDAGPU_EINVAL, "null context pointer");
    *out = nullptr;
    if (!pow2_in(i_max) || !pow2_in(j_max) || !pow2_in(l_max))
        return fail(DDAGPU_EINVAL, "lattice edges must be powers of two in [2, 128]");
    if (max_rhs < 1) return fail(DDAGPU_EINVAL, "max_rhs must be >= 1");
    if (!(kd > 0.0)) return fail(DDAGPU_EINVAL, "kd must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(DDAGPU_ENOTBUILT, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(DDAGPU_EINVAL, "bad device index");
    DevGuard dg(device);
    ddagpu_ctx *c = new ddagpu_ctx();
    c->dev = device;
    c->ni = i_max;
    c->nj = j_max;
    c->nl = l_max;
    c->N = (size_t)i_max * j_max * l_max;
    c->kd = kd;
    c->cap = max_rhs;
    c->tile_x = std::min(i_max <= 64 ? 32 : 16, 2 * l_max);
    c->rows_g = std::min(16, j_max);
    auto bail = [&](int code) {
        ddagpu_destroy(c);
        return code;
    };
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(DDAGPU_ECUDA, "stream creation failed"));
    const size_t n3 = 3 * c->N, wst = (size_t)3 * i_max * (2 * j_max) * (2 * l_max);
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t x) {
        if (x != cudaSuccess && e == cudaSuccess) e = x;
    };
    A(dalloc(&c->ahat, ahat_elems(i_max, j_max, l_max)));
    A(dalloc(&c->tw, (size_t)2 * (i_max + j_max + l_max)));
    A(dalloc(&c->work, wst * max_rhs));
    A(dalloc(&c->p, n3 * max_rhs));
    A(dalloc(&c->pmin, n3 * max_rhs));
    A(dalloc(&c->r, n3 * max_rhs));
    A(dalloc(&c->s, n3 * max_rhs));
    A(dalloc(&c->w, n3 * max_rhs));
    A(dalloc(&c->g, n3 * max_rhs));
    A(dalloc(&c->h, n3 * max_rhs));
    A(dalloc(&c->state, (size_t)max_rhs));
    A(dalloc(&c->active, (size_t)max_rhs));
    A(dalloc(&c->occ, c->N));
    A(dalloc(&c->step_dev, 1));
    A(dalloc(&c->nact_dev, (size_t)max_rhs));
    A(dalloc(&c->err_dev, 1));
    A(dalloc(&c->mv, (size_t)c->nmat_cap));
    A(dalloc(&c->alpha, (size_t)c->nmat_cap * max_rhs));
    A(dalloc(&c->kinc, (size_t)3 * max_rhs));
    A(dalloc(&c->einc, (size_t)6 * max_rhs));
    A(dalloc(&c->inc_tab, (size_t)(i_max + j_max + l_max) * max_rhs));
    A(dalloc(&c->cc_acc, (size_t)2 * max_rhs));
    A(dalloc(&c->cabs, (size_t)max_rhs));
    A(dalloc(&c->cext, (size_t)max_rhs));
    if (e != cudaSuccess)
        return bail(fail(e == cudaErrorMemoryAllocation ? DDAGPU_ENOMEM : DDAGPU_ECUDA,
                         std::string("allocation: ") + cudaGetErrorString(e)));
    std::vector<float2> tw((size_t)2 * (i_max + j_max + l_max));
    twiddles(i_max, tw.data());
    twiddles(j_max, tw.data() + 2 * i_max);
    twiddles(l_max, tw.data() + 2 * (i_max + j_max));
    c->L.ni = i_max;
    c->L.nj = j_max;
    c->L.nl = l_max;
    c->L.N = c->N;
    c->L.tw_i = c->tw;
    c->L.tw_j = c->tw + 2 * i_max;
    c->L.tw_l = c->tw + 2 * (i_max + j_max);
    if ((e = cudaMemcpyAsync(c->tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice,
                             c->st)) != cudaSuccess ||
        (e = matvec_prepare(c->L, c->tile_x, c->rows_g)) != cudaSuccess ||
        (matvec_fast_supported(c->L) && (e = matvec_fast_prepare(c->L)) != cudaSuccess) ||
        (e = post_prepare(j_max, l_max)) != cudaSuccess ||
        (e = green_build_octant(i_max, j_max, l_max, kd, c->ahat, c->st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->st)) != cudaSuccess)
        return bail(fail(DDAGPU_ECUDA, std::string("setup: ") + cudaGetErrorString(e)));
    c->fast = matvec_fast_supported(c->L) ? 1 : 0;
    if (c->fast) c->has_tmap = encode_work_maps(c);
    if (cudaMemset(c->err_dev, 0, sizeof(int)) != cudaSuccess)
        return bail(fail(DDAGPU_ECUDA, "setup: error flag"));
    *out = c;
    return DDAGPU_OK;
}

int ddagpu_destroy(ddagpu_ctx *c)
{
    if (!c) return DDAGPU_OK;
    DevGuard dg(c->dev);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->b32) cudaFree(c->b32);
    if (c->rb) cudaFree(c->rb);
    if (c->x64) cudaFree(c->x64);
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->wexec) cudaGraphExecDestroy(c->wexec);
    if (c->wgraph) cudaGraphDestroy(c->wgraph);
    void *ptrs[] = {c->ahat, c->tw,     c->work,   c->p,       c->pmin,   c->r,     c->s,
                    c->w,    c->g,      c->h,      c->state,   c->active, c->trace, c->occ,
                    c->mv,   c->alpha,  c->kinc,   c->einc,    c->ksc,    c->esc_acc,
                    c->cc_acc, c->normals, c->mueller, c->esc, c->cabs,   c->cext,
                    c->occ_b, c->ndip, c->step_dev, c->nact_dev, c->err_dev, c->worm_buf,
                    c->inc_tab, c->kz_tab, c->kz_val, c->kz_sum};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (c->pin) cudaFreeHost(c->pin);
    delete c->f64;
    delete c->mcg;
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return DDAGPU_OK;
}

int ddagpu_set_green(ddagpu_ctx *c, const float *cmA)
{
    if (!c || !cmA) return fail(DDAGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const size_t n = (size_t)8 * c->N * 6;
    float2 *dense = nullptr;
    CK(dalloc(&dense, n));
    cudaError_t e = cudaMemcpyAsync(dense, cmA, n * sizeof(float2), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = green_project_dense(c->ni, c->nj, c->nl, dense, c->ahat, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(dense);
    CK(e);
    return DDAGPU_OK;
}

void *ddagpu_stream(ddagpu_ctx *c) { return c ? (void *)c->st : nullptr; }

long long ddagpu_kernel_launches(ddagpu_ctx *c) { return c ? c->launches : -1; }

int ddagpu_set_tiling(ddagpu_ctx *c, int tile_x, int rows_g)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    int tx = tile_x ? tile_x : c->tile_x, rg = rows_g ? rows_g : c->rows_g;
    if (tx < 1 || (2 * c->nl) % tx != 0 || (tx & (tx - 1)) != 0)
        return fail(DDAGPU_EINVAL, "tile_x must be a power of two dividing 2 l_max");
    if (rg < 1 || c->nj % rg != 0 || (rg & (rg - 1)) != 0)
        return fail(DDAGPU_EINVAL, "rows_g must be a power of two dividing j_max");
    if (matvec_smem_x(c->L, tx) > 227 * 1024 || matvec_smem_yz(c->L, rg) > 227 * 1024)
        return fail(DDAGPU_EINVAL, "tiling exceeds shared memory");
    CK(matvec_prepare(c->L, tx, rg));
    c->tile_x = tx;
    c->rows_g = rg;
    return DDAGPU_OK;
}

int ddagpu_set_kernels(ddagpu_ctx *c, int fast)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    if (fast && !matvec_fast_supported(c->L))
        return fail(DDAGPU_EINVAL, "compile-time-sized passes need edges in {16, 32, 64, 128}");
    c->fast = fast ? 1 : 0;
    return DDAGPU_OK;
}

int ddagpu_get_kernels(ddagpu_ctx *c) { return c ? c->fast : -1; }

int ddagpu_get_tiling(ddagpu_ctx *c, int *tile_x, int *rows_g)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    if (tile_x) *tile_x = c->tile_x;
    if (rows_g) *rows_g = c->rows_g;
    return DDAGPU_OK;
}

int ddagpu_convolution_dev(ddagpu_ctx *c, const void *p_dev, void *out_dev, int nrhs, int conj)
{
    if (!c || !p_dev || !out_dev) return fail(DDAGPU_EINVAL, "null argument");
    if (nrhs < 1 || nrhs > c->cap) return fail(DDAGPU_EINVAL, "nrhs outside 1..max_rhs");
    DevGuard dg(c->dev);
    MatvecArgs a = mv_args(c, nrhs, (const float2 *)p_dev, (float2 *)out_dev, 0, 0.f, nullptr,
                           conj ? 1 : 0, 1, false);
    CK(launch_matvec(a, c->st));
    c->launches += 3;
    return DDAGPU_OK;
}

int ddagpu_autotune(ddagpu_ctx *c, int nrhs)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    if (nrhs < 1 || nrhs > c->cap) nrhs = std::min(c->cap, 4);
    DevGuard dg(c->dev);
    // candidates: x-pass columns per CTA and y/z staging rows
    std::vector<int> txs, rgs;
    for (int tx = 8; tx <= 64; tx *= 2)
        if ((2 * c->nl) % tx == 0 && matvec_smem_x(c->L, tx) <= 200 * 1024) txs.push_back(tx);
    for (int rg = 4; rg <= 32; rg *= 2)
        if (c->nj % rg == 0 && matvec_smem_yz(c->L, rg) <= 220 * 1024) rgs.push_back(rg);
    if (txs.empty() || rgs.empty()) return DDAGPU_OK;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto time_it = [&](float *ms) -> int {
        MatvecArgs a = mv_args(c, nrhs, c->p, c->r, 0, 0.f, nullptr, 0, 1, false);
        for (int k = 0; k < 2; k++) CK(launch_matvec(a, c->st));
        CK(cudaEventRecord(e0, c->st));
        for (int k = 0; k < 5; k++) CK(launch_matvec(a, c->st));
        CK(cudaEventRecord(e1, c->st));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(ms, e0, e1));
        return DDAGPU_OK;
    };
    float best = 1e30f;
    int btx = c->tile_x, brg = c->rows_g, bfast = 0;
    const int had_fast = c->fast;
    c->fast = 0;
    for (int tx : txs)
        for (int rg : rgs) {
            RET(ddagpu_set_tiling(c, tx, rg));
            float ms = 0;
            RET(time_it(&ms));
            if (ms < best) {
                best = ms;
                btx = tx;
                brg = rg;
            }
        }
    int bfx = 0, bfyz = 0;
    if (matvec_fast_supported(c->L)) {
        // the compile-time-sized passes in each launch variant
        c->fast = 1;
        for (int vx = 0; vx < (c->has_tmap ? kXVariants : 9); vx++)
            for (int vyz = 0; vyz < kYZVariants; vyz++) {
                c->fx = vx;
                c->fyz = vyz;
                float ms = 0;
                RET(time_it(&ms));
                if (ms < best) {
                    best = ms;
                    bfast = 1;
                    bfx = vx;
                    bfyz = vyz;
                }
            }
    }
    (void)had_fast;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->fast = 0;
    RET(ddagpu_set_tiling(c, btx, brg));
    c->fast = bfast;
    c->fx = bfx;
    c->fyz = bfyz;
    return DDAGPU_OK;
}

int ddagpu_convolution(ddagpu_ctx *c, const float *p, float *out, int conj)
{
    if (!c || !p || !out) return fail(DDAGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const size_t N = c->N;
    // AoS cvector -> SoA complex planes on the host side of the copy
    std::vector<float2> soa(3 * N);
    for (size_t q = 0; q < N; q++)
        for (int k = 0; k < 3; k++) soa[k * N + q] = make_float2(p[6 * q + 2 * k], p[6 * q + 2 * k + 1]);
    CK(cudaMemcpyAsync(c->p, soa.data(), 3 * N * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    MatvecArgs a = mv_args(c, 1, c->p, c->r, 0, 0.f, nullptr, conj ? 1 : 0, 1, false);
    CK(launch_matvec(a, c->st));
    CK(cudaMemcpyAsync(soa.data(), c->r, 3 * N * sizeof(float2), cudaMemcpyDeviceToHost, c->st));
    int werr = 0;
    CK(cudaMemcpyAsync(&werr, c->err_dev, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    RET(device_wait_error(c, werr));
    for (size_t q = 0; q < N; q++)
        for (int k = 0; k < 3; k++) {
            out[6 * q + 2 * k] = soa[k * N + q].x;
            out[6 * q + 2 * k + 1] = soa[k * N + q].y;
        }
    return DDAGPU_OK;
}

}  // extern "C"

namespace {

// Upload the per-solve material tables and occupancy; *nact (may be null) receives the
// active-cell count.  The reference calls DDA_FFT for both polarisations of a sample with
// the same occupancy, so an occupancy and material flags equal to the last ones uploaded
// (compared byte for byte) are neither checked, counted nor copied again.
int upload_materials(ddagpu_ctx *c, const int *mv, int nmat1, const signed char *occ,
                     int *nact = nullptr)
{
    if (nmat1 < 1 || nmat1 > c->nmat_cap) return fail(DDAGPU_EINVAL, "n_mat outside 0..254");
    c->occ_valid = false;
    CK(cudaMemcpyAsync(c->mv, mv, nmat1 * sizeof(int), cudaMemcpyHostToDevice, c->st));
    const bool same = c->occ_host.size() == c->N && c->mv_host.size() == (size_t)nmat1 &&
                      std::memcmp(c->mv_host.data(), mv, nmat1 * sizeof(int)) == 0 &&
                      std::memcmp(c->occ_host.data(), occ, c->N) == 0;
    if (!same) {
        c->occ_host.clear();
        RET(check_occ(occ, c->N, nmat1));
        CK(cudaMemcpyAsync(c->occ, occ, c->N, cudaMemcpyHostToDevice, c->st));
        c->occ_host_nact = count_active(occ, c->N, mv, nmat1);
        c->occ_host.assign(occ, occ + c->N);
        c->mv_host.assign(mv, mv + nmat1);
    }
    if (nact) *nact = c->occ_host_nact;
    return DDAGPU_OK;
}

// Uploads the scattering directions ks [nrhs][ndir][3] (pinned or pageable host memory)
// and plans the far field's kz groups for them; the group tables grow here, outside any
// graph capture, and a grown table drops the recorded graphs (they hold its address).
// nact: active cells per right-hand side, for the choice between the two forms.
int upload_directions(ddagpu_ctx *c, const double *ks, int nrhs, int ndir, bool pairs, double nact)
{
    c->kz.groups = 0;
    if (ndir <= 0) return DDAGPU_OK;
    CK(cudaMemcpyAsync(c->ksc, ks, (size_t)nrhs * ndir * 3 * sizeof(double), cudaMemcpyHostToDevice, c->st));
    plan_kz_groups(ks, nrhs, ndir, pairs, c->ni, c->nj, c->nl, nact, c->ff_mode, c->kz);
    if (!c->kz.groups) return DDAGPU_OK;
    auto grow = [&](auto *&buf, size_t &cap, size_t need) -> int {
        if (need <= cap) return DDAGPU_OK;
        drop_graphs(c);
        CK(cudaStreamSynchronize(c->st));
        cudaFree(buf);
        buf = nullptr;
        cap = 0;
        CK(dalloc(&buf, need));
        cap = need;
        return DDAGPU_OK;
    };
    RET(grow(c->kz_tab, c->kz_tab_cap, c->kz.tab.size()));
    RET(grow(c->kz_val, c->kz_val_cap, c->kz.kz.size()));
    RET(grow(c->kz_sum, c->kz_sum_cap, c->kz.sum_elems));
    CK(cudaMemcpyAsync(c->kz_tab, c->kz.tab.data(), c->kz.tab.size() * sizeof(int), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->kz_val, c->kz.kz.data(), c->kz.kz.size() * sizeof(double), cudaMemcpyHostToDevice,
                       c->st));
    return DDAGPU_OK;
}

// pairs: right-hand sides 2k and 2k+1 are the two polarisations of one orientation
int run_post(ddagpu_ctx *c, int nrhs, int nmat1, double d0, int ndir, bool pairs = false)
{
    PostArgs pa{};
    pa.pairs = pairs ? 1 : 0;
    pa.N = c->N;
    pa.nrhs = nrhs;
    pa.ni = c->ni;
    pa.nj = c->nj;
    pa.nl = c->nl;
    pa.occ = c->occ_stride ? c->occ_b : c->occ;
    pa.occ_stride = c->occ_stride;
    pa.mv = c->mv;
    pa.alpha = c->alpha;
    pa.nmat1 = nmat1;
    pa.p = c->p;
    pa.kinc = c->kinc;
    pa.einc = c->einc;
    pa.d0 = d0;
    pa.ndir = ndir;
    pa.ksc = c->ksc;
    pa.esc_acc = c->esc_acc;
    pa.cc_acc = c->cc_acc;
    if (ndir > 0 && c->kz.groups > 0) {
        pa.kz_groups = c->kz.groups;
        pa.kz_items = c->kz.items;
        pa.kz_slice = c->kz.slice;
        pa.kz_stride = c->kz.stride;
        pa.kz_tab = c->kz_tab;
        pa.kz_val = c->kz_val;
        pa.kz_sum = c->kz_sum;
    }
    int nk = 0;
    CK(launch_post(pa, c->esc, c->cabs, c->cext, c->st, &nk));
    c->launches += nk;
    return DDAGPU_OK;
}

// ---- batched solves: shared set-up and one chunk of up to cap / 2 orientations
struct BatchGeom {
    int nA = 0, nP = 0, ndir = 0, nmat1 = 0;
    std::vector<int> mv;
    std::vector<double> ksc0, nrm0;   // scattering directions and plane normals before rotation
};

int batch_check(ddagpu_ctx *c, const ddagpu_batch_cfg *cfg)
{
    if (c->cap < 2) return fail(DDAGPU_EINVAL, "the context needs max_rhs >= 2");
    if (cfg->n_mat < 1 || !cfg->m || cfg->nplanes < 1 || !(cfg->theta_step > 0.f))
        return fail(DDAGPU_EINVAL, "bad batch configuration");
    if (cfg->n_mat + 1 > c->nmat_cap) return fail(DDAGPU_EINVAL, "n_mat outside 0..254");
    if (cfg->polarizability < 1 || cfg->polarizability > 5)
        return fail(DDAGPU_EINVAL, "polarizability must be 1..5");
    return DDAGPU_OK;
}

int batch_setup(ddagpu_ctx *c, const ddagpu_batch_cfg *cfg, BatchGeom &g)
{
    g.nA = ddagpu_num_angles(cfg->theta_min, cfg->theta_max, cfg->theta_step);
    g.nP = cfg->nplanes;
    g.ndir = g.nA * g.nP;
    g.nmat1 = cfg->n_mat + 1;
    if (g.nA < 1) return fail(DDAGPU_EINVAL, "no scattering angles");
    RET(ensure_post(c, g.ndir, g.nP, g.nA));
    // material activity (main.cpp:610-613)
    g.mv.assign((size_t)g.nmat1, 0);
    for (int k = 0; k < cfg->n_mat; k++)
        g.mv[(size_t)k + 1] = (cfg->m[2 * k] == 1.f && cfg->m[2 * k + 1] == 0.f) ? 0 : 1;
    // scattering geometry before rotation (main.cpp:336-387)
    const double pi = 3.14159265358979323846264338327950288;
    g.ksc0.assign((size_t)g.ndir * 3, 0.0);
    g.nrm0.assign((size_t)g.nP * 3, 0.0);
    for (int pl = 0; pl < g.nP; pl++) {
        const double ang = pl * (180.0 / g.nP) * pi / 180.0, cs = std::cos(ang), sn = std::sin(ang);
        g.nrm0[3 * pl + 0] = sn;
        g.nrm0[3 * pl + 1] = cs;
        g.nrm0[3 * pl + 2] = 0.0;
        for (int a = 0; a < g.nA; a++) {
            const double th = ((double)cfg->theta_min + (double)cfg->theta_step * a) * pi / 180.0;
            const double k0[3] = {std::sin(th), 0.0, std::cos(th)};
            double *k = g.ksc0.data() + 3 * ((size_t)pl * g.nA + a);
            k[0] = cs * k0[0] + sn * k0[1];
            k[1] = -sn * k0[0] + cs * k0[1];
            k[2] = k0[2];
        }
    }
    return DDAGPU_OK;
}

// rot[o0 .. o0 + no) or, without rotations, the fixed orientation psi = iota = kappa = 0
void batch_rotations(const double *rot, int o0, int no, std::vector<double> &out)
{
    out.assign((size_t)9 * no, 0.0);
    for (int o = 0; o < no; o++)
        for (int q = 0; q < 9; q++)
            out[(size_t)9 * o + q] = rot ? rot[9 * ((size_t)o0 + o) + q] : (q % 4 == 0 ? 1.0 : 0.0);
}

int ensure_occ_batch(ddagpu_ctx *c)
{
    if (!c->occ_b) CK(dalloc(&c->occ_b, (size_t)c->cap * c->N));
    if (!c->ndip) CK(dalloc(&c->ndip, (size_t)c->cap));
    return DDAGPU_OK;
}

// Rasterises realisations r0 .. r0 + no of a monomer list into the context's batch
// occupancy (both polarisations of realisation k at right-hand sides 2k, 2k + 1) and
// returns their dipole counts (ndip, may be null) and active cells per right-hand side.
int agglomerate_rasterize(ddagpu_ctx *c, const BatchGeom &g, const float *monomers, const int *counts,
                          const std::vector<size_t> &first, int r0, int no, int *ndip,
                          std::vector<int> &nact)
{
    const size_t N = c->N;
    for (int k = 0; k < no; k++) {
        const int r = r0 + k;
        const size_t need = anthrax_scratch_bytes(counts[r]);
        if (need > c->worm_bytes) {   // grow the context's monomer buffer (stream-ordered)
            CK(cudaStreamSynchronize(c->st));
            cudaFree(c->worm_buf);
            c->worm_buf = nullptr;
            c->worm_bytes = 0;
            CK(cudaMalloc(&c->worm_buf, need));
            c->worm_bytes = need;
        }
        CK(anthrax_rasterize(monomers + 13 * first[(size_t)r], counts[r], c->ni, c->nj, c->nl,
                             c->occ_b + 2 * k * N, c->ndip + k, c->st, c->worm_buf, c->worm_bytes));
        CK(cudaMemcpyAsync(c->occ_b + (2 * k + 1) * N, c->occ_b + 2 * k * N, N,
                           cudaMemcpyDeviceToDevice, c->st));
        c->launches += 1;
    }
    std::vector<int> nd((size_t)no, 0);
    CK(cudaMemcpyAsync(nd.data(), c->ndip, no * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    nact.assign((size_t)2 * no, 0);
    for (int k = 0; k < no; k++) {
        if (ndip) ndip[r0 + k] = nd[(size_t)k];
        nact[2 * k] = nact[2 * k + 1] = g.mv[1] ? nd[(size_t)k] : 0;
        if (nact[2 * k] == 0) return fail(DDAGPU_EINVAL, "a realisation has no active dipoles");
    }
    return DDAGPU_OK;
}


// Per-right-hand-side occupancy (c->occ_b) for the lifetime of the guard.
struct OccBatch {
    ddagpu_ctx *c;
    explicit OccBatch(ddagpu_ctx *cc) : c(cc) { c->occ_stride = c->N; }
    ~OccBatch() { c->occ_stride = 0; }
};

// Pinned staging of at least `bytes` (the stream is idle: every batched chunk ends with a
// synchronisation).
int ensure_pin(ddagpu_ctx *c, size_t bytes)
{
    if (bytes <= c->pin_bytes) return DDAGPU_OK;
    if (c->pin) cudaFreeHost(c->pin);
    c->pin = nullptr;
    c->pin_bytes = 0;
    CK(cudaHostAlloc((void **)&c->pin, bytes, cudaHostAllocDefault));
    c->pin_bytes = bytes;
    return DDAGPU_OK;
}

// Offsets of a batched chunk's pinned staging: inputs kin, ein, ks, nv (double), al
// (float2); outputs ca, ce (float), mo (double); every block 16-byte aligned.
struct ChunkLayout {
    size_t n_kin, n_ein, n_ks, n_nv, n_al, n_mo;
    size_t o_ein, o_ks, o_nv, o_al, o_ca, o_ce, o_mo, total;
    ChunkLayout(int no, int ndir, int nP, int nA, int nmat1)
    {
        auto al16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
        const size_t nr = 2 * (size_t)no;
        n_kin = nr * 3;
        n_ein = nr * 6;
        n_ks = nr * ndir * 3;
        n_nv = (size_t)no * nP * 3;
        n_al = nr * nmat1;
        n_mo = (size_t)no * nA * 16;
        o_ein = al16(n_kin * 8);
        o_ks = o_ein + al16(n_ein * 8);
        o_nv = o_ks + al16(n_ks * 8);
        o_al = o_nv + al16(n_nv * 8);
        o_ca = o_al + al16(n_al * 8);
        o_ce = o_ca + al16(nr * 4);
        o_mo = o_ce + al16(nr * 4);
        total = o_mo + al16(n_mo * 8);
    }
};

// Results of a solved chunk: reads the outputs on the context's stream into cabs / cext /
// mueller (this chunk's first orientation) and the batch statistics.
int batch_chunk_finish(ddagpu_ctx *c, const BatchGeom &g, int no, const SolveResult &res,
                       double *cabs, double *cext, double *mueller, ddagpu_batch_info &bi)
{
    const int nr = 2 * no;
    const ChunkLayout Lc(no, g.ndir, g.nP, g.nA, g.nmat1);
    float *ca = (float *)(c->pin + Lc.o_ca), *ce = (float *)(c->pin + Lc.o_ce);
    double *mo = (double *)(c->pin + Lc.o_mo);
    CK(cudaMemcpyAsync(ca, c->cabs, nr * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(ce, c->cext, nr * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    if (mueller) CK(cudaMemcpyAsync(mo, c->mueller, Lc.n_mo * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int o = 0; o < no; o++) {
        if (cabs) cabs[o] = 0.5 * ca[(size_t)2 * o] + 0.5 * ca[(size_t)2 * o + 1];
        if (cext) cext[o] = 0.5 * ce[(size_t)2 * o] + 0.5 * ce[(size_t)2 * o + 1];
    }
    if (mueller) std::memcpy(mueller, mo, Lc.n_mo * sizeof(double));
    bi.n_rhs += nr;
    for (const RhsState &S : res.st) {
        bi.max_steps = std::max(bi.max_steps, S.steps);
        bi.rolled_back += S.restored;
        bi.max_err = std::max(bi.max_err, S.restored ? S.err_min : S.err);
    }
    return DDAGPU_OK;
}

// Solves no orientations (rotation matrices rot[no][9]) as 2 no right-hand sides -- both
// incident polarisations, x and y before rotation (main.cpp:153-154) -- whose occupancy is
// on the device, then far fields, cross sections and the Mueller matrices averaged over the
// planes (main.cpp:870-949).  cabs / cext / mueller point at this chunk's first orientation.
// With rec the chunk is only prepared (inputs uploaded, solve recorded into rec's graph if
// it has one) for a group launch; the group then calls batch_chunk_finish.
int batch_chunk(ddagpu_ctx *c, const ddagpu_batch_cfg *cfg, const BatchGeom &g, const double *rot,
                int no, int nact, const int *nact_per, double *cabs, double *cext, double *mueller,
                ddagpu_batch_info &bi, GroupRecord *rec = nullptr)
{
    const int nr = 2 * no, ndir = g.ndir, nP = g.nP, nA = g.nA, nmat1 = g.nmat1;
    const double d0 = c->kd;
    const ChunkLayout Lc(no, ndir, nP, nA, nmat1);
    RET(ensure_pin(c, Lc.total));
    double *kin = (double *)c->pin, *ein = (double *)(c->pin + Lc.o_ein), *ks = (double *)(c->pin + Lc.o_ks),
           *nv = (double *)(c->pin + Lc.o_nv);
    float2 *al = (float2 *)(c->pin + Lc.o_al);
    std::memset(c->pin, 0, Lc.o_ca);
    for (int o = 0; o < no; o++) {
        const double *T = rot + 9 * (size_t)o;
        auto R = [&](const double *v, double *out) {
            for (int i = 0; i < 3; i++) out[i] = T[3 * i] * v[0] + T[3 * i + 1] * v[1] + T[3 * i + 2] * v[2];
        };
        const double kz[3] = {0, 0, 1}, ex[3] = {1, 0, 0}, ey[3] = {0, 1, 0};
        double k[3], e0[3], e1[3];
        R(kz, k);
        R(ex, e0);
        R(ey, e1);
        for (int q = 0; q < 2; q++) {
            const int rr = 2 * o + q;
            const double *e = q ? e1 : e0;
            for (int i = 0; i < 3; i++) {
                kin[3 * rr + i] = k[i];
                ein[6 * rr + 2 * i] = e[i];
                ein[6 * rr + 2 * i + 1] = 0.0;
            }
            for (int dd = 0; dd < ndir; dd++)
                R(g.ksc0.data() + 3 * dd, ks + ((size_t)rr * ndir + dd) * 3);
            for (int mm = 0; mm < cfg->n_mat; mm++) {
                const cd a = polarizability(cfg->polarizability, d0, {cfg->m[2 * mm], cfg->m[2 * mm + 1]},
                                            kin + 3 * rr, ein + 6 * rr);
                al[(size_t)rr * nmat1 + mm + 1] = make_float2((float)a.r, (float)a.i);
            }
        }
        for (int pl = 0; pl < nP; pl++) R(g.nrm0.data() + 3 * pl, nv + ((size_t)o * nP + pl) * 3);
    }
    CK(cudaMemcpyAsync(c->kinc, kin, Lc.n_kin * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->einc, ein, Lc.n_ein * sizeof(double), cudaMemcpyHostToDevice, c->st));
    double nact_mean = nact;
    if (nact_per) {
        nact_mean = 0.0;
        for (int r = 0; r < nr; r++) nact_mean += nact_per[r];
        nact_mean /= nr;
    }
    RET(upload_directions(c, ks, nr, ndir, true, nact_mean));
    CK(cudaMemcpyAsync(c->normals, nv, Lc.n_nv * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->alpha, al, Lc.n_al * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    SolveResult res;
    // far field, cross sections and the plane-averaged Mueller matrices, after the solve
    // (recorded with it when the solve is one graph launch)
    const std::function<int()> post = [&]() -> int {
        RET(run_post(c, nr, nmat1, d0, ndir, true));
        MuellerArgs m{no, nP, nA, ndir, c->kinc, c->einc, c->ksc, c->normals, c->esc, c->mueller};
        CK(launch_mueller(m, c->st));
        c->launches += 1;
        return DDAGPU_OK;
    };
    c->post_key = ((long long)ndir << 40) | ((long long)no << 24) | ((long long)nP << 12) | nA;
    // both polarisations of every orientation with the same polarisabilities (every model
    // but LDR): step 0 transforms one scalar field per orientation (MatvecArgs::pair)
    bool same = true;
    for (int o = 0; o < no && same; o++)
        same = std::memcmp(al + (size_t)2 * o * nmat1, al + (size_t)(2 * o + 1) * nmat1,
                           nmat1 * sizeof(float2)) == 0;
    c->pair_step0 = same ? 1 : 0;
    const int rc = run_solver(c, nr, cfg->solver, cfg->tau, cfg->max_step, cfg->err_max, nmat1, d0, nact,
                              res, false, nullptr, nact_per, &post, rec);
    c->pair_step0 = 0;
    RET(rc);
    if (rec) return DDAGPU_OK;
    return batch_chunk_finish(c, g, no, res, cabs, cext, mueller, bi);
}

}  // namespace

extern "C" {

int ddagpu_dda_fft(ddagpu_ctx *c, int iNoIllumination, int solver, float rTau, int i_max,
                   int j_max, int l_max, const float *cListMaterials, const int *iListMV, int n_mat,
                   const signed char *cAlpha, int Max_Step, float Error_max, float d0,
                   const float *kinc, const float *Einc, int iMode_FFT, int iNoScPl, int iNoA,
                   const float *ksc, float *Esc, float *rCabs, float *rCext,
                   ddagpu_solve_info *info, double *trace)
{
    (void)iNoIllumination;
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    if (i_max != c->ni || j_max != c->nj || l_max != c->nl)
        return fail(DDAGPU_EMISMATCH, "The workspace does not match the lattice dimensions");
    if (!cListMaterials || !iListMV || !cAlpha || !kinc || !Einc || !rCabs || !rCext)
        return fail(DDAGPU_EINVAL, "null argument");
    if (iMode_FFT != 0 && iMode_FFT != 1) return fail(DDAGPU_EINVAL, "iMode_FFT must be 0 or 1");
    if (iNoScPl < 0 || iNoA < 0 || ((size_t)iNoScPl * iNoA > 0 && (!ksc || !Esc)))
        return fail(DDAGPU_EINVAL, "bad scattering directions");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const int nmat1 = n_mat + 1, ndir = iNoScPl * iNoA;
    int nact = 0;
    RET(upload_materials(c, iListMV, nmat1, cAlpha, &nact));
    RET(ensure_post(c, std::max(ndir, 1), std::max(iNoScPl, 1), std::max(iNoA, 1)));
    std::vector<float2> al((size_t)nmat1);
    for (int m = 0; m < nmat1; m++) al[(size_t)m] = make_float2(cListMaterials[2 * m], cListMaterials[2 * m + 1]);
    double kd3[3] = {kinc[0], kinc[1], kinc[2]};
    double ed6[6];
    for (int k = 0; k < 6; k++) ed6[k] = Einc[k];
    std::vector<double> kd((size_t)ndir * 3);
    for (size_t k = 0; k < kd.size(); k++) kd[k] = ksc[k];
    CK(cudaMemcpyAsync(c->alpha, al.data(), nmat1 * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->kinc, kd3, sizeof kd3, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->einc, ed6, sizeof ed6, cudaMemcpyHostToDevice, c->st));
    RET(upload_directions(c, kd.data(), 1, ndir, false, nact));
    // nact: counted by upload_materials
    if (nact == 0) return fail(DDAGPU_EINVAL, "no active dipoles");
    SolveResult res;
    RET(run_solver(c, 1, solver, rTau, Max_Step, Error_max, nmat1, d0, nact, res, trace != nullptr));
    RET(run_post(c, 1, nmat1, d0, ndir));
    std::vector<float2> esc((size_t)ndir * 3);
    float ca = 0, ce = 0;
    if (ndir) CK(cudaMemcpyAsync(esc.data(), c->esc, esc.size() * sizeof(float2), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&ca, c->cabs, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&ce, c->cext, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (size_t k = 0; k < esc.size(); k++) {
        Esc[2 * k] = esc[k].x;
        Esc[2 * k + 1] = esc[k].y;
    }
    *rCabs = ca;
    *rCext = ce;
    const RhsState &S = res.st[0];
    if (info) {
        info->steps = S.steps;
        info->step_min = S.step_min;
        info->rolled_back = S.restored;
        info->matvecs = res.matvec0 + res.matvec_it * S.steps;
        info->err = S.err;
        info->err_min = S.err_min;
    }
    if (trace)
        for (int k = 0; k <= Max_Step; k++) trace[k] = k <= S.steps ? res.trace[(size_t)k] : 0.0;
    return DDAGPU_OK;
}

}  // extern "C"
namespace {

// Outer refinement loop for one right-hand side already in c->b32 (see
// ddagpu_dda_fft_refined); leaves p = float(x64).
int refine_loop(ddagpu_ctx *c, int solver, float rTau, int nmat1, double d0, int nact,
                double Error_max, int max_outer, double inner_rel, int inner_max_step,
                ddagpu_refine_info &ri, double &err)
{
    FieldArgs F = fa_args(c, 1, nmat1, d0, rTau);
    {
        int one = 1;
        CK(cudaMemcpyAsync(c->active, &one, sizeof one, cudaMemcpyHostToDevice, c->st));
    }
    CK(launch_refine(0, F, c->st));
    c->launches += 1;
    std::memset(&ri, 0, sizeof ri);
    err = 0.0;
    for (int k = 0;; k++) {
        // true residual in FP64: r = b - (x - alpha G*x), G*x from the float matvec
        CK(launch_refine(3, F, c->st));
        CK(launch_matvec(mv_args(c, 1, c->p, c->w, 0, 0.f, nullptr, 0, nmat1, false), c->st));
        const double zero8[kAcc] = {0, 0, 0, 0, 0, 0, 0, 0};
        double *acc_dev = reinterpret_cast<double *>(reinterpret_cast<char *>(c->state) +
                                                     offsetof(RhsState, acc));
        CK(cudaMemcpyAsync(acc_dev, zero8, sizeof zero8, cudaMemcpyHostToDevice, c->st));
        int one = 1;
        CK(cudaMemcpyAsync(c->active, &one, sizeof one, cudaMemcpyHostToDevice, c->st));
        CK(launch_refine(1, F, c->st));
        c->launches += 5;
        double acc = 0.0;
        CK(cudaMemcpyAsync(&acc, acc_dev, sizeof acc, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        err = acc / nact;
        if (k < 64) ri.err_history[k] = err;
        ri.outer = k;
        if (err <= Error_max || k >= max_outer) break;
        // inner FP32 solve of A d = r from d0 = r, to a fraction of the current error
        SolveResult res;
        const float inner_err = (float)std::max(inner_rel * err, 0.5 * Error_max);
        RET(run_solver(c, 1, solver, rTau, inner_max_step, inner_err, nmat1, d0, nact, res, false, c->rb));
        ri.inner_steps += res.st[0].steps;
        ri.matvecs += res.matvec0 + res.matvec_it * res.st[0].steps;
        CK(cudaMemcpyAsync(c->active, &one, sizeof one, cudaMemcpyHostToDevice, c->st));
        CK(launch_refine(2, F, c->st));
        c->launches += 1;
    }
    ri.err = err;
    ri.matvecs += ri.outer + 1;
    CK(launch_refine(3, F, c->st));
    c->launches += 1;
    return DDAGPU_OK;
}

// Refinement of CG (solver 0): the reference's CG recurrences with FP64 fields, scalars and
// true residuals around the FP32 FFT matvec, never restarted (mixed_cg, fp64.cu).  The
// right-hand side is p_inc in FP64 (kinc, einc) or, with from_b32, the float field in
// c->b32.  Leaves float(x) in c->p.
int mixed_refine(ddagpu_ctx *c, const float *cListMaterials, int nmat1, int nact, double d0,
                 const double *kinc, const double *einc, bool from_b32, double Error_max,
                 int max_outer, double inner_rel, int inner_max_step, ddagpu_refine_info &ri)
{
    if (!c->mcg) c->mcg = new MixedCgBuffers();
    CK(c->mcg->ensure(3 * c->N));
    std::vector<double2> al((size_t)nmat1);
    for (int m = 0; m < nmat1; m++) al[(size_t)m] = make_double2(cListMaterials[2 * m], cListMaterials[2 * m + 1]);
    CK(cudaMemcpyAsync(c->mcg->alpha, al.data(), nmat1 * sizeof(double2), cudaMemcpyHostToDevice, c->st));
    Field64View f{c->N, c->ni, c->nj, c->nl, c->occ, c->mv, c->mcg->alpha};
    CK(f64_right_hand_side(f, d0, kinc, einc, from_b32 ? c->b32 : nullptr, c->mcg->b, c->st));
    c->launches += 1;
    const ConvFn conv = [&](const float2 *src, float2 *out) {
        c->launches += 3;
        return launch_matvec(mv_args(c, 1, src, out, 0, 0.f, nullptr, 0, nmat1, false), c->st);
    };
    MixedCgResult R;
    CK(mixed_cg(*c->mcg, f, al.data(), nmat1, nact, Error_max, max_outer, inner_rel, inner_max_step,
                conv, c->s, c->w, c->rb, c->p, c->st, R, &c->launches));
    std::memset(&ri, 0, sizeof ri);
    ri.outer = R.outer;
    ri.inner_steps = R.iterations;
    ri.matvecs = R.matvecs;
    ri.err = R.err;
    for (int k = 0; k < 64; k++) ri.err_history[k] = R.history[k];
    int werr = 0;
    CK(cudaMemcpyAsync(&werr, c->err_dev, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    RET(device_wait_error(c, werr));
    return DDAGPU_OK;
}

void aos_to_soa(const float *in, float2 *out, size_t N)
{
    for (size_t q = 0; q < N; q++)
        for (int k = 0; k < 3; k++) out[k * N + q] = make_float2(in[6 * q + 2 * k], in[6 * q + 2 * k + 1]);
}

void soa_to_aos(const float2 *in, float *out, size_t N)
{
    for (size_t q = 0; q < N; q++)
        for (int k = 0; k < 3; k++) {
            out[6 * q + 2 * k] = in[k * N + q].x;
            out[6 * q + 2 * k + 1] = in[k * N + q].y;
        }
}

}  // namespace

extern "C" {

int ddagpu_solve_linear(ddagpu_ctx *c, int solver, float rTau, const float *cListMaterials,
                        const int *iListMV, int n_mat, const signed char *cAlpha, const float *rhs,
                        double Error_max, int max_step, int refine, double inner_rel,
                        int inner_max_step, float *x_out, ddagpu_refine_info *info)
{
    if (!c || !cListMaterials || !iListMV || !cAlpha || !rhs || !x_out)
        return fail(DDAGPU_EINVAL, "null argument");
    if (!(Error_max > 0.0) || max_step < 0 || (refine && (inner_max_step < 1 ||
                                                          !(inner_rel > 0.0 && inner_rel < 1.0))))
        return fail(DDAGPU_EINVAL, "bad solve parameters");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const int nmat1 = n_mat + 1;
    const size_t n3 = 3 * c->N;
    if (!c->b32) {
        CK(dalloc(&c->b32, n3));
        CK(dalloc(&c->rb, n3));
        CK(dalloc(&c->x64, n3));
    }
    int nact = 0;
    RET(upload_materials(c, iListMV, nmat1, cAlpha, &nact));
    std::vector<float2> al((size_t)nmat1);
    for (int m = 0; m < nmat1; m++) al[(size_t)m] = make_float2(cListMaterials[2 * m], cListMaterials[2 * m + 1]);
    CK(cudaMemcpyAsync(c->alpha, al.data(), nmat1 * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    // nact: counted by upload_materials
    if (nact == 0) return fail(DDAGPU_EINVAL, "no active dipoles");
    std::vector<float2> soa(n3);
    aos_to_soa(rhs, soa.data(), c->N);
    CK(cudaMemcpyAsync(c->b32, soa.data(), n3 * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    ddagpu_refine_info ri;
    std::memset(&ri, 0, sizeof ri);
    if (refine && solver == 0) {
        RET(mixed_refine(c, cListMaterials, nmat1, nact, c->kd, nullptr, nullptr, true, Error_max,
                         max_step, inner_rel, inner_max_step, ri));
    } else if (refine) {
        RhsState S0;
        std::memset(&S0, 0, sizeof S0);
        S0.active = 1;
        S0.nact = nact;
        CK(cudaMemcpyAsync(c->state, &S0, sizeof S0, cudaMemcpyHostToDevice, c->st));
        double err = 0.0;
        RET(refine_loop(c, solver, rTau, nmat1, c->kd, nact, Error_max, max_step, inner_rel,
                        inner_max_step, ri, err));
    } else {
        SolveResult res;
        RET(run_solver(c, 1, solver, rTau, max_step, (float)Error_max, nmat1, c->kd, nact, res,
                       false, c->b32));
        const RhsState &S = res.st[0];
        ri.outer = 0;
        ri.inner_steps = S.steps;
        ri.matvecs = res.matvec0 + res.matvec_it * S.steps;
        ri.err = S.restored ? S.err_min : S.err;
        ri.err_history[0] = ri.err;
    }
    CK(cudaMemcpyAsync(soa.data(), c->p, n3 * sizeof(float2), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    soa_to_aos(soa.data(), x_out, c->N);
    if (info) *info = ri;
    return DDAGPU_OK;
}

}  // extern "C"

extern "C" {

int ddagpu_dda_fft_refined(ddagpu_ctx *c, int solver, float rTau, const float *cListMaterials,
                           const int *iListMV, int n_mat, const signed char *cAlpha, float d0,
                           const float *kinc, const float *Einc, double Error_max, int max_outer,
                           double inner_rel, int inner_max_step, int iNoScPl, int iNoA,
                           const float *ksc, float *Esc, float *rCabs, float *rCext,
                           ddagpu_refine_info *info)
{
    if (!c || !cListMaterials || !iListMV || !cAlpha || !kinc || !Einc || !rCabs || !rCext)
        return fail(DDAGPU_EINVAL, "null argument");
    if (max_outer < 0 || inner_max_step < 1 || !(inner_rel > 0.0 && inner_rel < 1.0) ||
        !(Error_max > 0.0))
        return fail(DDAGPU_EINVAL, "bad refinement parameters");
    if (iNoScPl < 0 || iNoA < 0 || ((size_t)iNoScPl * iNoA > 0 && (!ksc || !Esc)))
        return fail(DDAGPU_EINVAL, "bad scattering directions");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const int nmat1 = n_mat + 1, ndir = iNoScPl * iNoA;
    const size_t n3 = 3 * c->N;
    if (!c->b32) {
        CK(dalloc(&c->b32, n3));
        CK(dalloc(&c->rb, n3));
        CK(dalloc(&c->x64, n3));
    }
    int nact = 0;
    RET(upload_materials(c, iListMV, nmat1, cAlpha, &nact));
    RET(ensure_post(c, std::max(ndir, 1), std::max(iNoScPl, 1), std::max(iNoA, 1)));
    std::vector<float2> al((size_t)nmat1);
    for (int m = 0; m < nmat1; m++) al[(size_t)m] = make_float2(cListMaterials[2 * m], cListMaterials[2 * m + 1]);
    double kd3[3] = {kinc[0], kinc[1], kinc[2]}, ed6[6];
    for (int k = 0; k < 6; k++) ed6[k] = Einc[k];
    std::vector<double> kdir((size_t)ndir * 3);
    for (size_t k = 0; k < kdir.size(); k++) kdir[k] = ksc[k];
    CK(cudaMemcpyAsync(c->alpha, al.data(), nmat1 * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->kinc, kd3, sizeof kd3, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->einc, ed6, sizeof ed6, cudaMemcpyHostToDevice, c->st));
    RET(upload_directions(c, kdir.data(), 1, ndir, false, nact));
    // nact: counted by upload_materials
    if (nact == 0) return fail(DDAGPU_EINVAL, "no active dipoles");
    ddagpu_refine_info ri;
    double err = 0.0;
    if (solver == 0) {
        RET(mixed_refine(c, cListMaterials, nmat1, nact, d0, kd3, ed6, false, Error_max, max_outer,
                         inner_rel, inner_max_step, ri));
    } else {
        // outer right-hand side b = p_inc (FirstApproximation), x = b
        {
            RhsState S0;
            std::memset(&S0, 0, sizeof S0);
            S0.active = 1;
            S0.nact = nact;
            int one = 1;
            CK(cudaMemcpyAsync(c->state, &S0, sizeof S0, cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(c->active, &one, sizeof one, cudaMemcpyHostToDevice, c->st));
        }
        FieldArgs F = fa_args(c, 1, nmat1, d0, rTau);
        CK(launch_first_approx(F, c->st));
        CK(cudaMemcpyAsync(c->b32, c->p, n3 * sizeof(float2), cudaMemcpyDeviceToDevice, c->st));
        c->launches += 1;
        RET(refine_loop(c, solver, rTau, nmat1, d0, nact, Error_max, max_outer, inner_rel,
                        inner_max_step, ri, err));
    }
    RET(run_post(c, 1, nmat1, d0, ndir));
    std::vector<float2> esc((size_t)ndir * 3);
    float ca = 0, ce = 0;
    if (ndir) CK(cudaMemcpyAsync(esc.data(), c->esc, esc.size() * sizeof(float2), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&ca, c->cabs, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&ce, c->cext, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (size_t k = 0; k < esc.size(); k++) {
        Esc[2 * k] = esc[k].x;
        Esc[2 * k + 1] = esc[k].y;
    }
    *rCabs = ca;
    *rCext = ce;
    if (info) *info = ri;
    return DDAGPU_OK;
}

int ddagpu_solve_fp64(ddagpu_ctx *c, int solver, double tau, const double *alpha,
                      const int *iListMV, int n_mat, const signed char *cAlpha, double d0,
                      const double *kinc, const double *Einc, const double *rhs, const double *x0,
                      int Max_Step, double Error_max, int ndir, const double *ksc, double *Esc,
                      double *Cabs, double *Cext, double *p_out, ddagpu_solve_info *info,
                      double *trace)
{
    if (!c || !alpha || !iListMV || !cAlpha || !kinc || !Einc || !Cabs || !Cext)
        return fail(DDAGPU_EINVAL, "null argument");
    if (solver < 0 || solver > 3) return fail(DDAGPU_EINVAL, "solver must be 0..3");
    if (Max_Step < 0 || ndir < 0 || (ndir > 0 && (!ksc || !Esc)))
        return fail(DDAGPU_EINVAL, "bad solve parameters");
    if (ndir > 65535) return fail(DDAGPU_EINVAL, "at most 65535 directions per FP64 solve");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const int nmat1 = n_mat + 1;
    int nact = 0;
    RET(upload_materials(c, iListMV, nmat1, cAlpha, &nact));
    if (nact == 0) return fail(DDAGPU_EINVAL, "no active dipoles");
    if (!c->f64) c->f64 = new Fp64Buffers();
    CK(c->f64->ensure(c->ni, c->nj, c->nl, c->kd, c->st));
    const size_t N = c->N;
    // the reference's cvector layout [N][3] <-> structure of arrays [3][N]
    auto to_soa = [&](const double *in, std::vector<double2> &out) {
        out.resize(3 * N);
        for (size_t q = 0; q < N; q++)
            for (int k = 0; k < 3; k++) out[k * N + q] = make_double2(in[6 * q + 2 * k], in[6 * q + 2 * k + 1]);
    };
    std::vector<double2> al((size_t)nmat1), rs, xs, ps;
    for (int m = 0; m < nmat1; m++) al[(size_t)m] = make_double2(alpha[2 * m], alpha[2 * m + 1]);
    if (rhs) to_soa(rhs, rs);
    if (x0) to_soa(x0, xs);
    if (p_out) ps.resize(3 * N);
    Fp64Problem P{};
    P.solver = solver;
    P.tau = tau;
    P.nmat1 = nmat1;
    P.alpha = al.data();
    P.occ = c->occ;
    P.mv = c->mv;
    P.nact = nact;
    P.d0 = d0;
    for (int k = 0; k < 3; k++) P.kinc[k] = kinc[k];
    for (int k = 0; k < 6; k++) P.einc[k] = Einc[k];
    P.rhs = rhs ? rs.data() : nullptr;
    P.x0 = x0 ? xs.data() : nullptr;
    P.max_step = Max_Step;
    P.err_max = Error_max;
    P.ndir = ndir;
    P.ksc = ksc;
    Fp64Result R;
    R.esc = Esc;
    R.p = p_out ? ps.data() : nullptr;
    R.trace = trace;
    R.trace_len = trace ? Max_Step + 1 : 0;
    if (trace) std::fill(trace, trace + Max_Step + 1, 0.0);
    CK(solve_fp64(*c->f64, P, c->st, R, &c->launches));
    *Cabs = R.cabs;
    *Cext = R.cext;
    if (p_out)
        for (size_t q = 0; q < N; q++)
            for (int k = 0; k < 3; k++) {
                p_out[6 * q + 2 * k] = ps[k * N + q].x;
                p_out[6 * q + 2 * k + 1] = ps[k * N + q].y;
            }
    if (info) {
        info->steps = R.steps;
        info->step_min = R.step_min;
        info->rolled_back = R.rolled_back;
        info->matvecs = R.matvecs;
        info->err = R.err;
        info->err_min = R.err_min;
    }
    return DDAGPU_OK;
}

int ddagpu_release_fp64(ddagpu_ctx *c)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    if (c->st) cudaStreamSynchronize(c->st);
    delete c->f64;
    c->f64 = nullptr;
    return DDAGPU_OK;
}

int ddagpu_farfield(ddagpu_ctx *c, const int *iListMV, int n_mat, const signed char *cAlpha,
                    float d0, const float *p, int ndir, const float *ksc, float *Esc)
{
    if (!c || !iListMV || !cAlpha || !p || (ndir > 0 && (!ksc || !Esc)) || ndir < 0)
        return fail(DDAGPU_EINVAL, "null or bad argument");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const int nmat1 = n_mat + 1;
    int nact = 0;
    RET(upload_materials(c, iListMV, nmat1, cAlpha, &nact));
    RET(ensure_post(c, std::max(ndir, 1), 1, 1));
    const size_t N = c->N;
    std::vector<float2> soa(3 * N);
    for (size_t q = 0; q < N; q++)
        for (int k = 0; k < 3; k++) soa[k * N + q] = make_float2(p[6 * q + 2 * k], p[6 * q + 2 * k + 1]);
    CK(cudaMemcpyAsync(c->p, soa.data(), 3 * N * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    std::vector<double> kd((size_t)ndir * 3);
    for (size_t k = 0; k < kd.size(); k++) kd[k] = ksc[k];
    std::vector<float2> zero_alpha((size_t)nmat1, make_float2(0.f, 0.f));
    double z6[6] = {1, 0, 0, 0, 0, 0}, z3[3] = {0, 0, 1};
    CK(cudaMemcpyAsync(c->alpha, zero_alpha.data(), nmat1 * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->kinc, z3, sizeof z3, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->einc, z6, sizeof z6, cudaMemcpyHostToDevice, c->st));
    RET(upload_directions(c, kd.data(), 1, ndir, false, nact));
    RET(run_post(c, 1, nmat1, d0, ndir));
    std::vector<float2> esc((size_t)ndir * 3);
    if (ndir) CK(cudaMemcpyAsync(esc.data(), c->esc, esc.size() * sizeof(float2), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (size_t k = 0; k < esc.size(); k++) {
        Esc[2 * k] = esc[k].x;
        Esc[2 * k + 1] = esc[k].y;
    }
    return DDAGPU_OK;
}

int ddagpu_cabscext(ddagpu_ctx *c, float d0, const float *kinc, const float *Einc,
                    const float *cListMaterials, int n_mat, const signed char *cAlpha,
                    const float *p, float *Cabs, float *Cext)
{
    if (!c || !kinc || !Einc || !cListMaterials || !cAlpha || !p || !Cabs || !Cext)
        return fail(DDAGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const int nmat1 = n_mat + 1;
    std::vector<int> mv((size_t)nmat1, 1);
    RET(upload_materials(c, mv.data(), nmat1, cAlpha));
    RET(ensure_post(c, 1, 1, 1));
    const size_t N = c->N;
    std::vector<float2> soa(3 * N);
    for (size_t q = 0; q < N; q++)
        for (int k = 0; k < 3; k++) soa[k * N + q] = make_float2(p[6 * q + 2 * k], p[6 * q + 2 * k + 1]);
    CK(cudaMemcpyAsync(c->p, soa.data(), 3 * N * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    std::vector<float2> al((size_t)nmat1);
    for (int m = 0; m < nmat1; m++) al[(size_t)m] = make_float2(cListMaterials[2 * m], cListMaterials[2 * m + 1]);
    double kd3[3] = {kinc[0], kinc[1], kinc[2]}, ed6[6];
    for (int k = 0; k < 6; k++) ed6[k] = Einc[k];
    CK(cudaMemcpyAsync(c->alpha, al.data(), nmat1 * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->kinc, kd3, sizeof kd3, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->einc, ed6, sizeof ed6, cudaMemcpyHostToDevice, c->st));
    RET(run_post(c, 1, nmat1, d0, 0));
    CK(cudaMemcpyAsync(Cabs, c->cabs, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(Cext, c->cext, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return DDAGPU_OK;
}

int ddagpu_mueller(ddagpu_ctx *c, const float *kinc, const float *einc0, const float *einc1,
                   int nplanes, int nangles, const float *ksc, const float *normals,
                   const float *esc0, const float *esc1, float *out)
{
    if (!c || !kinc || !einc0 || !einc1 || !ksc || !normals || !esc0 || !esc1 || !out ||
        nplanes < 1 || nangles < 1)
        return fail(DDAGPU_EINVAL, "null or bad argument");
    if (c->cap < 2) return fail(DDAGPU_EINVAL, "the context needs max_rhs >= 2");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    const int ndir = nplanes * nangles;
    RET(ensure_post(c, ndir, nplanes, nangles));
    std::vector<double> kd(6), ed(12), ks((size_t)2 * ndir * 3), nv((size_t)nplanes * 3);
    for (int k = 0; k < 3; k++) kd[k] = kd[3 + k] = kinc[k];
    for (int k = 0; k < 6; k++) {
        ed[k] = einc0[k];
        ed[6 + k] = einc1[k];
    }
    for (int k = 0; k < ndir * 3; k++) ks[k] = ks[(size_t)ndir * 3 + k] = ksc[k];
    for (int k = 0; k < nplanes * 3; k++) nv[k] = normals[k];
    std::vector<float2> es((size_t)2 * ndir * 3);
    for (int k = 0; k < ndir * 3; k++) {
        es[k] = make_float2(esc0[2 * k], esc0[2 * k + 1]);
        es[(size_t)ndir * 3 + k] = make_float2(esc1[2 * k], esc1[2 * k + 1]);
    }
    CK(cudaMemcpyAsync(c->kinc, kd.data(), kd.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->einc, ed.data(), ed.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->ksc, ks.data(), ks.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->normals, nv.data(), nv.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->esc, es.data(), es.size() * sizeof(float2), cudaMemcpyHostToDevice, c->st));
    MuellerArgs m{1, nplanes, nangles, ndir, c->kinc, c->einc, c->ksc, c->normals, c->esc, c->mueller};
    CK(launch_mueller(m, c->st));
    std::vector<double> mo((size_t)nangles * 16);
    CK(cudaMemcpyAsync(mo.data(), c->mueller, mo.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (size_t k = 0; k < mo.size(); k++) out[k] = (float)mo[k];
    return DDAGPU_OK;
}

int ddagpu_farfield_noalloc(int device, int i_max, int j_max, int l_max, float d0,
                            const signed char *occ_dev, const int *mv_dev, int n_mat,
                            const void *p_dev, int ndir, const float *ksc_dev, float *esc_dev,
                            void *stream)
{
    if (!pow2_in(i_max) || !pow2_in(j_max) || !pow2_in(l_max))
        return fail(DDAGPU_EINVAL, "lattice edges must be powers of two in [2, 128]");
    if (n_mat < 0 || n_mat + 1 > kMaxMaterials + 1) return fail(DDAGPU_EINVAL, "n_mat outside 0..255");
    if (ndir < 0 || ndir > farfield_noalloc_max_dirs())
        return fail(DDAGPU_EINVAL, "ndir exceeds the allocation-free maximum of " +
                                       std::to_string(farfield_noalloc_max_dirs()) + " directions");
    if (ndir == 0) return DDAGPU_OK;
    if (!occ_dev || !mv_dev || !p_dev || !ksc_dev || !esc_dev)
        return fail(DDAGPU_EINVAL, "null device pointer");
    DevGuard dg(device);
    double *scratch = nullptr;
    CK(farfield_noalloc_scratch(device, &scratch));
    PostArgs a{};
    a.N = (size_t)i_max * j_max * l_max;
    a.nrhs = 1;
    a.ni = i_max;
    a.nj = j_max;
    a.nl = l_max;
    a.occ = occ_dev;
    a.mv = mv_dev;
    a.nmat1 = n_mat + 1;   // cells whose material index exceeds n_mat count as empty
    a.p = (const float2 *)p_dev;
    a.d0 = d0;
    a.ndir = ndir;
    CK(farfield_noalloc(a, ksc_dev, (float2 *)esc_dev, scratch, (cudaStream_t)stream));
    return DDAGPU_OK;
}

int ddagpu_mc_rotations(unsigned long long base_seed, int worker, int count, double *rot)
{
    if (!rot || count < 0 || worker < 0) return fail(DDAGPU_EINVAL, "bad argument");
    // per-worker stream (main.cpp:803-804), xorshift64* (randomize.cpp:44-58)
    unsigned long long s = base_seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(worker + 1);
    if (!s) s = 0x9E3779B97F4A7C15ULL;
    auto next = [&]() {
        s ^= s >> 12;
        s ^= s << 25;
        s ^= s >> 27;
        return (double)(int)((s * 2685821657736338717ULL) >> 33);
    };
    const double pi = 3.14159265358979323846264338327950288, RMAX = 2147483647.0;
    for (int k = 0; k < count; k++) {
        // Euler draw and rotation matrix, main.cpp:876-898
        const double cps = next() * 2.0 / RMAX - 1.0, psi = std::acos(cps), sps = std::sin(psi);
        const double io = next() * 2.0 * pi / RMAX, ka = next() * 2.0 * pi / RMAX;
        const double cio = std::cos(io), sio = std::sin(io), cka = std::cos(ka), ska = std::sin(ka);
        double *t = rot + 9 * (size_t)k;
        t[0] = cio * cka - cps * sio * ska;
        t[1] = sio * cka + cps * cio * ska;
        t[2] = sps * ska;
        t[3] = -cio * ska - cps * sio * cka;
        t[4] = -sio * ska + cps * cio * cka;
        t[5] = sps * cka;
        t[6] = sps * sio;
        t[7] = -sps * cio;
        t[8] = cps;
    }
    return DDAGPU_OK;
}

unsigned long long ddagpu_rng_seed(unsigned long long base_seed, int worker)
{
    const unsigned long long s = base_seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(worker + 1);
    return s ? s : 0x9E3779B97F4A7C15ULL;   // dda_srand, randomize.cpp:44-48
}

long long ddagpu_anthrax_count(int i_max, int j_max, int l_max, float packing,
                               float monomer_radius, float length_ratio)
{
    return anthrax_count(i_max, j_max, l_max, packing, monomer_radius, length_ratio);
}

int ddagpu_anthrax_place(unsigned long long *rng_state, int i_max, float monomer_radius,
                         float monomer_length, int count, float *monomers)
{
    if (!rng_state || !monomers || count < 1 || i_max < 2 || !(monomer_radius > 0.f))
        return fail(DDAGPU_EINVAL, "bad agglomerate arguments");
    const long long max_tries = 2000000LL + 20000LL * count;
    if (anthrax_place(rng_state, i_max, monomer_radius, monomer_length, count, monomers, max_tries))
        return fail(DDAGPU_EINVAL, "monomer placement did not finish (packing too dense)");
    return DDAGPU_OK;
}

int ddagpu_anthrax_rasterize(int device, int i_max, int j_max, int l_max, const float *monomers,
                             int count, signed char *occ, int *ndip)
{
    if (!pow2_in(i_max) || !pow2_in(j_max) || !pow2_in(l_max))
        return fail(DDAGPU_EINVAL, "lattice edges must be powers of two in [2, 128]");
    if (!monomers || !occ || count < 0) return fail(DDAGPU_EINVAL, "null or bad argument");
    DevGuard dg(device);
    const size_t N = (size_t)i_max * j_max * l_max;
    cudaStream_t st;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    signed char *d = nullptr;
    int *nd = nullptr, h = 0;
    cudaError_t e = cudaMallocAsync(&d, N, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&nd, sizeof(int), st);
    if (e == cudaSuccess) e = anthrax_rasterize(monomers, count, i_max, j_max, l_max, d, nd, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(occ, d, N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, nd, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (d) cudaFreeAsync(d, st);
    if (nd) cudaFreeAsync(nd, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    CK(e);
    CK(e2);
    if (ndip) *ndip = h;
    return DDAGPU_OK;
}

int ddagpu_set_fast_variant(ddagpu_ctx *c, int x_variant, int yz_variant)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    if (x_variant < 0 || x_variant >= kXVariants || yz_variant < 0 || yz_variant >= kYZVariants)
        return fail(DDAGPU_EINVAL, "launch variants: x 0..11, y/z 0..2");
    if (x_variant >= 9 && !c->has_tmap) return fail(DDAGPU_EINVAL, "no tensor maps on this device");
    std::lock_guard<std::mutex> lk(c->mu);
    c->fx = x_variant;
    c->fyz = yz_variant;
    return DDAGPU_OK;
}

int ddagpu_farfield_plan(const double *ksc, int nrhs, int ndir, int pairs, int ni, int nj, int nl,
                         double nact, int mode, int *groups, int *items)
{
    if (!groups || nrhs < 0 || ndir < 0 || (nrhs > 0 && ndir > 0 && !ksc) || ni < 1 || nj < 1 || nl < 1 ||
        mode < 0 || mode > 2)
        return fail(DDAGPU_EINVAL, "bad far-field plan arguments");
    KzPlan P;
    plan_kz_groups(ksc, nrhs, ndir, pairs != 0, ni, nj, nl, nact, mode, P);
    *groups = P.groups;
    if (items) *items = P.groups ? P.items : 0;
    return DDAGPU_OK;
}

int ddagpu_set_farfield_mode(ddagpu_ctx *c, int mode)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    if (mode < 0 || mode > 2) return fail(DDAGPU_EINVAL, "far-field mode 0..2");
    std::lock_guard<std::mutex> lk(c->mu);
    c->ff_mode = mode;
    return DDAGPU_OK;
}

int ddagpu_get_fast_variant(ddagpu_ctx *c, int *x_variant, int *yz_variant)
{
    if (!c || !x_variant || !yz_variant) return fail(DDAGPU_EINVAL, "null argument");
    *x_variant = c->fx;
    *yz_variant = c->fyz;
    return DDAGPU_OK;
}

int ddagpu_selftest_wait_timeout(ddagpu_ctx *c, int on)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    std::lock_guard<std::mutex> lk(c->mu);
    c->wait_selftest = on ? 1 : 0;
    drop_graphs(c);   // recorded launches hold the old setting
    return DDAGPU_OK;
}

int ddagpu_set_solver_graph(ddagpu_ctx *c, int on)
{
    if (!c) return fail(DDAGPU_EINVAL, "null context");
    std::lock_guard<std::mutex> lk(c->mu);
    c->graph_on = on ? 1 : 0;
    return DDAGPU_OK;
}

long long ddagpu_solver_graph_runs(ddagpu_ctx *c) { return c ? c->graph_runs : -1; }

int ddagpu_random_ellipsoid_seeds(unsigned long long *rng_state, int i_max, int j_max, int l_max,
                                  float b_a, float c_a, int n_seeds, float *seeds)
{
    if (!rng_state || !seeds || n_seeds < 1 || i_max < 1 || j_max < 1 || l_max < 1)
        return fail(DDAGPU_EINVAL, "bad random-ellipsoid arguments");
    if (random_ellipsoid_seeds(rng_state, i_max, j_max, l_max, b_a, c_a, n_seeds, seeds))
        return fail(DDAGPU_EINVAL, "the ellipsoid does not fit in the lattice");
    return DDAGPU_OK;
}

int ddagpu_random_ellipsoid_fill(int device, int i_max, int j_max, int l_max, float b_a, float c_a,
                                 const float *seeds, const int *seeds_per_material, int n_mat,
                                 signed char *occ, int *ndip)
{
    if (!seeds || !seeds_per_material || !occ || n_mat < 1 || n_mat > kMaxMaterials - 1 ||
        i_max < 1 || j_max < 1 || l_max < 1)
        return fail(DDAGPU_EINVAL, "bad random-ellipsoid arguments");
    long long total = 0;
    for (int m = 0; m < n_mat; m++) {
        if (seeds_per_material[m] < 0) return fail(DDAGPU_EINVAL, "negative seed count");
        total += seeds_per_material[m];
    }
    if (total < 1 || total > (1 << 24)) return fail(DDAGPU_EINVAL, "bad total seed count");
    if ((float)i_max * b_a > (float)j_max || (float)i_max * c_a > (float)l_max)
        return fail(DDAGPU_EINVAL, "the ellipsoid does not fit in the lattice");
    DevGuard dg(device);
    const size_t N = (size_t)i_max * j_max * l_max;
    cudaStream_t st;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    signed char *dv = nullptr;
    int *nd = nullptr, h = 0;
    cudaError_t e = cudaMallocAsync(&dv, N, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&nd, sizeof(int), st);
    if (e == cudaSuccess)
        e = random_ellipsoid_fill(seeds, seeds_per_material, n_mat, i_max, j_max, l_max, b_a, c_a, dv,
                                  nd, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(occ, dv, N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, nd, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (dv) cudaFreeAsync(dv, st);
    if (nd) cudaFreeAsync(nd, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    CK(e);
    CK(e2);
    if (ndip) *ndip = h;
    return DDAGPU_OK;
}

int ddagpu_fixed_rotation(double psi, double iota, double kappa, double *rot)
{
    if (!rot) return fail(DDAGPU_EINVAL, "null argument");
    // Z(-psi), then Y(-iota), then X(-kappa) (main.cpp:516-541, Rotation_* dda_func.cpp:7-34)
    const double d = 3.14159265358979323846264338327950288 / 180.0;
    const double a = -psi * d, b = -iota * d, g = -kappa * d;
    const double Z[9] = {std::cos(a), std::sin(a), 0, -std::sin(a), std::cos(a), 0, 0, 0, 1};
    const double Y[9] = {std::cos(b), 0, -std::sin(b), 0, 1, 0, std::sin(b), 0, std::cos(b)};
    const double X[9] = {1, 0, 0, 0, std::cos(g), std::sin(g), 0, -std::sin(g), std::cos(g)};
    double YZ[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            YZ[3 * i + j] = 0;
            for (int k = 0; k < 3; k++) YZ[3 * i + j] += Y[3 * i + k] * Z[3 * k + j];
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            rot[3 * i + j] = 0;
            for (int k = 0; k < 3; k++) rot[3 * i + j] += X[3 * i + k] * YZ[3 * k + j];
        }
    return DDAGPU_OK;
}

int ddagpu_orientation_solves(ddagpu_ctx *c, const ddagpu_batch_cfg *cfg, int n_orient,
                              const double *rot, double *cabs, double *cext, double *mueller,
                              ddagpu_batch_info *info)
{
    if (!c || !cfg || !rot || n_orient < 0) return fail(DDAGPU_EINVAL, "null or bad argument");
    RET(batch_check(c, cfg));
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    BatchGeom g;
    RET(batch_setup(c, cfg, g));
    // occupancy shared by every orientation
    int nact = 0;
    if (cfg->occ) {
        RET(upload_materials(c, g.mv.data(), g.nmat1, cfg->occ, &nact));
        c->occ_valid = true;
        c->occ_nmat1 = g.nmat1;
        c->occ_nact = nact;
    } else {
        // occupancy of the previous batched call, still on the device
        if (!c->occ_valid || c->occ_nmat1 != g.nmat1)
            return fail(DDAGPU_EINVAL, "cfg->occ is null and no occupancy is resident");
        CK(cudaMemcpyAsync(c->mv, g.mv.data(), g.nmat1 * sizeof(int), cudaMemcpyHostToDevice, c->st));
        nact = c->occ_nact;
    }
    if (nact == 0) return fail(DDAGPU_EINVAL, "no active dipoles");
    const int per = c->cap / 2;
    ddagpu_batch_info bi{0, 0, 0, 0.0};
    for (int o0 = 0; o0 < n_orient; o0 += per) {
        const int no = std::min(per, n_orient - o0);
        RET(batch_chunk(c, cfg, g, rot + 9 * (size_t)o0, no, nact, nullptr, cabs ? cabs + o0 : nullptr,
                        cext ? cext + o0 : nullptr,
                        mueller ? mueller + (size_t)o0 * g.nA * 16 : nullptr, bi));
    }
    if (info) *info = bi;
    return DDAGPU_OK;
}

int ddagpu_realization_solves(ddagpu_ctx *c, const ddagpu_batch_cfg *cfg, int n_real,
                              const signed char *occ, const double *rot, double *cabs,
                              double *cext, double *mueller, ddagpu_batch_info *info)
{
    if (!c || !cfg || !occ || n_real < 0) return fail(DDAGPU_EINVAL, "null or bad argument");
    RET(batch_check(c, cfg));
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    BatchGeom g;
    RET(batch_setup(c, cfg, g));
    RET(ensure_occ_batch(c));
    const size_t N = c->N;
    for (int k = 0; k < n_real; k++) RET(check_occ(occ + (size_t)k * N, N, g.nmat1));
    CK(cudaMemcpyAsync(c->mv, g.mv.data(), g.nmat1 * sizeof(int), cudaMemcpyHostToDevice, c->st));
    const int per = c->cap / 2;
    ddagpu_batch_info bi{0, 0, 0, 0.0};
    std::vector<int> nact;
    std::vector<double> rots;
    for (int o0 = 0; o0 < n_real; o0 += per) {
        const int no = std::min(per, n_real - o0);
        nact.assign((size_t)2 * no, 0);
        for (int k = 0; k < no; k++) {
            const signed char *src = occ + (size_t)(o0 + k) * N;
            nact[2 * k] = nact[2 * k + 1] = count_active(src, N, g.mv.data(), g.nmat1);
            if (nact[2 * k] == 0) return fail(DDAGPU_EINVAL, "a realisation has no active dipoles");
            CK(cudaMemcpyAsync(c->occ_b + 2 * k * N, src, N, cudaMemcpyHostToDevice, c->st));
            CK(cudaMemcpyAsync(c->occ_b + (2 * k + 1) * N, c->occ_b + 2 * k * N, N,
                               cudaMemcpyDeviceToDevice, c->st));
        }
        batch_rotations(rot, o0, no, rots);
        OccBatch ob(c);
        RET(batch_chunk(c, cfg, g, rots.data(), no, 0, nact.data(), cabs ? cabs + o0 : nullptr,
                        cext ? cext + o0 : nullptr,
                        mueller ? mueller + (size_t)o0 * g.nA * 16 : nullptr, bi));
    }
    if (info) *info = bi;
    return DDAGPU_OK;
}

int ddagpu_agglomerate_solves(ddagpu_ctx *c, const ddagpu_batch_cfg *cfg, int n_real,
                              const float *monomers, const int *counts, const double *rot,
                              double *cabs, double *cext, double *mueller, int *ndip,
                              ddagpu_batch_info *info)
{
    if (!c || !cfg || !counts || n_real < 0) return fail(DDAGPU_EINVAL, "null or bad argument");
    RET(batch_check(c, cfg));
    if (cfg->n_mat != 1) return fail(DDAGPU_EINVAL, "agglomerates are one material (n_mat = 1)");
    std::vector<size_t> first((size_t)n_real + 1, 0);
    for (int k = 0; k < n_real; k++) {
        if (counts[k] < 0) return fail(DDAGPU_EINVAL, "negative monomer count");
        first[(size_t)k + 1] = first[(size_t)k] + (size_t)counts[k];
    }
    if (first[(size_t)n_real] && !monomers) return fail(DDAGPU_EINVAL, "null monomers");
    std::lock_guard<std::mutex> lk(c->mu);
    DevGuard dg(c->dev);
    BatchGeom g;
    RET(batch_setup(c, cfg, g));
    RET(ensure_occ_batch(c));
    const size_t N = c->N;
    CK(cudaMemcpyAsync(c->mv, g.mv.data(), g.nmat1 * sizeof(int), cudaMemcpyHostToDevice, c->st));
    const int per = c->cap / 2;
    ddagpu_batch_info bi{0, 0, 0, 0.0};
    std::vector<int> nact;
    std::vector<double> rots;
    for (int o0 = 0; o0 < n_real; o0 += per) {
        const int no = std::min(per, n_real - o0);
        RET(agglomerate_rasterize(c, g, monomers, counts, first, o0, no, ndip, nact));
        batch_rotations(rot, o0, no, rots);
        OccBatch ob(c);
        RET(batch_chunk(c, cfg, g, rots.data(), no, 0, nact.data(), cabs ? cabs + o0 : nullptr,
                        cext ? cext + o0 : nullptr,
                        mueller ? mueller + (size_t)o0 * g.nA * 16 : nullptr, bi));
    }
    if (info) *info = bi;
    return DDAGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- groups of contexts
// Lattices of different sizes solved as ONE graph launch: every member context's whole
// batched solve is an independent branch of one graph (its state set-up, step 0, its own
// conditional while loop, rollback, far field and Mueller matrices), recorded once per
// solve shape and replayed.  The members' inputs are uploaded on their own streams, which
// the group's stream waits for before the launch; the members' streams wait for the
// launch before the results are read.
struct ddagpu_group {
    std::vector<ddagpu_ctx *> ctx;
    int dev = 0;
    cudaStream_t st = nullptr;
    std::vector<cudaEvent_t> ev;          // one per member: its inputs are uploaded
    cudaEvent_t done = nullptr;           // the launch has finished
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<char> used;               // members with a branch in the graph
    std::vector<ddagpu_ctx::GraphKey> keys;
    std::vector<long long> gens;
    std::vector<GroupRecord> rec;         // per member: kernel counts of its branch
    long long runs = 0;
    std::mutex mu;
};


extern "C" {

int ddagpu_group_create(ddagpu_group **out, ddagpu_ctx *const *ctxs, int nctx)
{
    if (!out || !ctxs || nctx < 1) return fail(DDAGPU_EINVAL, "null or bad argument");
    *out = nullptr;
    for (int k = 0; k < nctx; k++) {
        if (!ctxs[k]) return fail(DDAGPU_EINVAL, "null context");
        if (ctxs[k]->dev != ctxs[0]->dev) return fail(DDAGPU_EINVAL, "group members on different devices");
        for (int q = 0; q < k; q++)
            if (ctxs[q] == ctxs[k]) return fail(DDAGPU_EINVAL, "a context appears twice in the group");
    }
    DevGuard dg(ctxs[0]->dev);
    ddagpu_group *g = new ddagpu_group();
    g->ctx.assign(ctxs, ctxs + nctx);
    g->dev = ctxs[0]->dev;
    g->ev.assign((size_t)nctx, nullptr);
    cudaError_t e = cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking);
    for (int k = 0; k < nctx && e == cudaSuccess; k++)
        e = cudaEventCreateWithFlags(&g->ev[(size_t)k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        ddagpu_group_destroy(g);
        return fail(DDAGPU_ECUDA, std::string("group set-up: ") + cudaGetErrorString(e));
    }
    *out = g;
    return DDAGPU_OK;
}

int ddagpu_group_destroy(ddagpu_group *g)
{
    if (!g) return DDAGPU_OK;
    DevGuard dg(g->dev);
    if (g->st) cudaStreamSynchronize(g->st);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    for (cudaEvent_t e : g->ev)
        if (e) cudaEventDestroy(e);
    if (g->done) cudaEventDestroy(g->done);
    if (g->st) cudaStreamDestroy(g->st);
    delete g;
    return DDAGPU_OK;
}

long long ddagpu_group_graph_runs(ddagpu_group *g) { return g ? g->runs : -1; }

int ddagpu_group_agglomerate_solves(ddagpu_group *grp, const ddagpu_batch_cfg *cfg, const int *n_real,
                                    const float *const *monomers, const int *const *counts,
                                    const double *const *rot, double *const *cabs, double *const *cext,
                                    double *const *mueller, int *const *ndip, ddagpu_batch_info *info)
{
    if (!grp || !cfg || !n_real || !monomers || !counts) return fail(DDAGPU_EINVAL, "null or bad argument");
    const int nctx = (int)grp->ctx.size();
    std::lock_guard<std::mutex> glk(grp->mu);
    std::vector<std::unique_lock<std::mutex>> locks;
    std::vector<BatchGeom> geo((size_t)nctx);
    std::vector<std::vector<double>> rots((size_t)nctx);
    std::vector<std::vector<int>> nact((size_t)nctx);
    std::vector<char> used((size_t)nctx, 0);
    for (int k = 0; k < nctx; k++) {
        ddagpu_ctx *c = grp->ctx[(size_t)k];
        RET(batch_check(c, cfg));
        if (cfg->n_mat != 1) return fail(DDAGPU_EINVAL, "agglomerates are one material (n_mat = 1)");
        if (n_real[k] < 0 || n_real[k] > c->cap / 2)
            return fail(DDAGPU_EINVAL, "a member's realisations exceed its max_rhs / 2 (one batch per member)");
        used[(size_t)k] = n_real[k] > 0;
        for (int r = 0; r < n_real[k]; r++)
            if (counts[k][r] < 0) return fail(DDAGPU_EINVAL, "negative monomer count");
    }
    // members locked in address order: groups sharing contexts cannot deadlock
    std::vector<ddagpu_ctx *> order(grp->ctx);
    std::sort(order.begin(), order.end());
    for (ddagpu_ctx *m : order) locks.emplace_back(m->mu);
    DevGuard dg(grp->dev);
    std::vector<ddagpu_batch_info> bi((size_t)nctx, ddagpu_batch_info{0, 0, 0, 0.0});
    // ---- inputs of every member on its own stream, and the key of its solve
    std::vector<GroupRecord> rec((size_t)nctx);
    for (int k = 0; k < nctx; k++) {
        if (!used[(size_t)k]) continue;
        ddagpu_ctx *c = grp->ctx[(size_t)k];
        const int no = n_real[k];
        std::vector<size_t> first((size_t)no + 1, 0);
        for (int r = 0; r < no; r++) first[(size_t)r + 1] = first[(size_t)r] + (size_t)counts[k][r];
        if (first[(size_t)no] && !monomers[k]) return fail(DDAGPU_EINVAL, "null monomers");
        BatchGeom &g = geo[(size_t)k];
        RET(batch_setup(c, cfg, g));
        RET(ensure_occ_batch(c));
        CK(cudaMemcpyAsync(c->mv, g.mv.data(), g.nmat1 * sizeof(int), cudaMemcpyHostToDevice, c->st));
        RET(agglomerate_rasterize(c, g, monomers[k], counts[k], first, 0, no, ndip ? ndip[k] : nullptr,
                                  nact[(size_t)k]));
        batch_rotations(rot ? rot[k] : nullptr, 0, no, rots[(size_t)k]);
        OccBatch ob(c);
        RET(batch_chunk(c, cfg, g, rots[(size_t)k].data(), no, 0, nact[(size_t)k].data(), nullptr, nullptr,
                        nullptr, bi[(size_t)k], &rec[(size_t)k]));
    }
    // ---- the group's graph: rebuilt when a member's solve shape or buffers change
    bool rebuild = !grp->exec || grp->used != used;
    for (int k = 0; k < nctx && !rebuild; k++)
        if (used[(size_t)k] && (std::memcmp(&rec[(size_t)k].key, &grp->keys[(size_t)k], sizeof(ddagpu_ctx::GraphKey)) ||
                                grp->gens[(size_t)k] != grp->ctx[(size_t)k]->gen))
            rebuild = true;
    if (rebuild) {
        if (grp->exec) cudaGraphExecDestroy(grp->exec);
        if (grp->graph) cudaGraphDestroy(grp->graph);
        grp->exec = nullptr;
        grp->graph = nullptr;
        cudaGraph_t G = nullptr;
        CK(cudaGraphCreate(&G, 0));
        int rc = DDAGPU_OK;
        for (int k = 0; k < nctx && rc == DDAGPU_OK; k++) {
            if (!used[(size_t)k]) continue;
            ddagpu_ctx *c = grp->ctx[(size_t)k];
            rec[(size_t)k].graph = G;
            OccBatch ob(c);
            rc = batch_chunk(c, cfg, geo[(size_t)k], rots[(size_t)k].data(), n_real[k], 0, nact[(size_t)k].data(),
                             nullptr, nullptr, nullptr, bi[(size_t)k], &rec[(size_t)k]);
        }
        cudaGraphExec_t x = nullptr;
        const cudaError_t e = rc == DDAGPU_OK ? cudaGraphInstantiate(&x, G, 0) : cudaSuccess;
        if (rc != DDAGPU_OK || e != cudaSuccess) {
            cudaGraphDestroy(G);
            if (rc != DDAGPU_OK) return rc;
            return fail(DDAGPU_ECUDA, std::string("group graph (instantiate): ") + cudaGetErrorString(e));
        }
        grp->graph = G;
        grp->exec = x;
        grp->used = used;
        grp->keys.assign((size_t)nctx, ddagpu_ctx::GraphKey{});
        grp->gens.assign((size_t)nctx, 0);
        grp->rec = rec;
        for (int k = 0; k < nctx; k++) {
            grp->keys[(size_t)k] = rec[(size_t)k].key;
            grp->gens[(size_t)k] = grp->ctx[(size_t)k]->gen;
            grp->rec[(size_t)k].graph = nullptr;
        }
    }
    // ---- one launch for every member
    for (int k = 0; k < nctx; k++) {
        if (!used[(size_t)k]) continue;
        CK(cudaEventRecord(grp->ev[(size_t)k], grp->ctx[(size_t)k]->st));
        CK(cudaStreamWaitEvent(grp->st, grp->ev[(size_t)k], 0));
    }
    CK(cudaGraphLaunch(grp->exec, grp->st));
    CK(cudaEventRecord(grp->done, grp->st));
    grp->runs += 1;
    for (int k = 0; k < nctx; k++) {
        if (!used[(size_t)k]) continue;
        ddagpu_ctx *c = grp->ctx[(size_t)k];
        CK(cudaStreamWaitEvent(c->st, grp->done, 0));
        SolveResult res;
        const GroupRecord &R = grp->rec[(size_t)k];
        RET(read_whole_solve(c, 2 * n_real[k], res, R.n_fixed, R.n_per_iter, R.matvec0, R.matvec_it, false));
        RET(batch_chunk_finish(c, geo[(size_t)k], n_real[k], res, cabs ? cabs[k] : nullptr,
                               cext ? cext[k] : nullptr, mueller ? mueller[k] : nullptr, bi[(size_t)k]));
    }
    if (info)
        for (int k = 0; k < nctx; k++) info[k] = bi[(size_t)k];
    return DDAGPU_OK;
}

}  // extern "C"
