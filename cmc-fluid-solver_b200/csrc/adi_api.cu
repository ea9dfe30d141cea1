// C ABI of libadi_b200.so (include/adi_b200.h): handle lifetime, device memory,
// mask upload and checks, segment building and the time-step schedule.
//
// The schedule is the CPU backend's (AdiSolver3D.cpp:306-391 with SolveDirection
// :564-666): per global iteration Z (cur -> next), Y (next -> half),
// X (half -> next), each repeated num_local times with the nonlinear merge
// temp = (temp + result)/2 after every sweep, plus one more merge after X.  The
// merges are fused into the sweeps; the nonlinear layer is double buffered so that
// every sweep sees the pre-merge layer, as the reference's separate merge pass
// guarantees.  Layers are swapped by index, as the reference swaps pointers.
#include "adi_b200.h"
#include "adi_internal.cuh"

#include <type_traits>

#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <initializer_list>
#include <new>
#include <string>
#include <vector>

using namespace adi;

struct adi_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int prec = ADI_FP32;
    int solver = ADI_SOLVER_FAST;
    int nx = 0, ny = 0, nz = 0;
    long long n = 0;
    double dx = 0, dy = 0, dz = 0;
    adi_fluid_params params{};

    uint8_t *d_code = nullptr;
    void *d_nv[4] = {};
    void *d_L[5][4] = {};  // five layers of four fields
    int cur = 0, nxt = 1, half = 2, ta = 3, tb = 4;

    int *d_line_lo[3] = {}, *d_line_hi[3] = {};
    int32_t *d_segs[3] = {};
    long long nsegs[3] = {0, 0, 0};
    void *d_scratch = nullptr;
    size_t scratch_bytes = 0;

    int *d_err = nullptr;   // raised by a device-side bounded wait that gave up
    double *d_psum = nullptr, *d_sum = nullptr;
    unsigned long long *d_pcnt = nullptr, *d_cnt = nullptr;

    // built-in profiler (adi_set_profiling / adi_get_profile)
    struct Rec {
        int cls;
        cudaEvent_t a, b;
    };
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_free;
    std::vector<Rec> ev_pending;
    int64_t launches[ADI_K_NUM] = {};
    double ms[ADI_K_NUM] = {};
    int64_t bytes[ADI_K_NUM] = {};
    long long seg_nodes[3] = {0, 0, 0};
    FastShape shape[3] = {{4, 8, 0}, {4, 8, 0}, {4, 8, 0}};
    bool tuned = false;

    bool mask_set = false, segs_built = false, contract_ok = false;
    bool bv_synced = false;   // cur == node values at every BOUND/VALVE node
    int fault = ADI_FAULT_NONE;   // adi_set_fault_injection

    // Step results the host reads back: divergence sum and count, the device error
    // flag, the residual maxima (bit patterns).  Pinned, so the copies can sit in a
    // captured graph.
    struct Pinned {
        double sum;
        unsigned long long cnt;
        int err;
        int pad;
        unsigned long long res[2];
    };
    Pinned *h_pin = nullptr;
    unsigned long long *d_res = nullptr;

    // CUDA graphs of whole steps, one per (dt, iteration counts, error flag,
    // boundary update, layer roles); replayed by adi_step / adi_time_step / adi_run.
    struct GraphEntry {
        uint64_t key[4];
        cudaGraphExec_t exec;
        int post_ta, post_tb;
        int64_t launches[ADI_K_NUM];
        int64_t bytes[ADI_K_NUM];
    };
    std::vector<GraphEntry> graphs;
    bool graphs_on = true;
    cudaStream_t cap_stream = nullptr;
    // pipelined host I/O (adi_step_io): upload and download streams, one event per
    // downloaded piece, the result's device copy that the download reads
    static constexpr int IO_PIECES = 4;   // pieces per field
    cudaStream_t io_up = nullptr, io_down = nullptr;
    cudaEvent_t ev_io_up = nullptr, ev_io_ready = nullptr, ev_io_down = nullptr;
    cudaEvent_t ev_io_piece[4 * IO_PIECES] = {};
    void *d_io[4] = {};
    bool io_used = false;
    int adjoint_K = -4;  // adjoint sweep: chunk length (< 0: split solve + accumulation); 0: one thread per line
    // adjoint workspace (checkpoints, tape, adjoint layers), kept between
    // adi_adjoint_run calls and grown when a call needs more; freed by adi_destroy
    char *adj_mem = nullptr;
    size_t adj_cap = 0;
    char *mask_mem = nullptr;   // scratch of the mask builders and adi_get_layer, kept between calls
    size_t mask_cap = 0;
    std::string contract_msg;
    std::string err;
    double diff_error = 0.0;
    long long num_in = 0;
};

namespace {

const char *kVersion = "adi_b200 1.0 (sm_100a)";

adi_status fail(adi_handle *h, adi_status s, const std::string &msg)
{
    if (h) h->err = msg;
    return s;
}

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(h, ADI_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
    } while (0)

size_t esize(const adi_handle *h) { return h->prec == ADI_FP64 ? 8 : 4; }

template <typename R>
DomainView<R> view(const adi_handle *h)
{
    DomainView<R> d;
    d.nx = h->nx; d.ny = h->ny; d.nz = h->nz; d.n = h->n;
    d.code = h->d_code;
    for (int v = 0; v < 4; v++) d.nv[v] = (const R *)h->d_nv[v];
    return d;
}

template <typename R>
Layer<R> layer(const adi_handle *h, int l)
{
    Layer<R> x;
    for (int v = 0; v < 4; v++) x.f[v] = (R *)h->d_L[l][v];
    return x;
}

template <typename R>
CLayer<R> clayer(const adi_handle *h, int l)
{
    CLayer<R> x;
    for (int v = 0; v < 4; v++) x.f[v] = (const R *)h->d_L[l][v];
    return x;
}

// Scalar constants of one sweep, in the working precision, with BuildMatrix's
// operations (AdiSolver3D.cpp:744-752: vis/(h*h); :761,775,789: 3/dt + 2*vis;
// (2*h) denominators).  Host code is compiled with -ffp-contract=off.
template <typename R>
SweepConst<R> sweep_const(const adi_handle *h, int dir, R dt)
{
    SweepConst<R> k;
    const R dx = (R)h->dx, dy = (R)h->dy, dz = (R)h->dz;
    const R hh = dir == 0 ? dx : (dir == 1 ? dy : dz);
    const R v_vis = (R)h->params.v_vis, t_vis = (R)h->params.t_vis;
    k.three = R(3);
    k.dt = dt;
    k.two_h = R(2) * hh;
    k.vis_v = v_vis / (hh * hh);
    k.vis_t = t_vis / (hh * hh);
    k.b_v = R(3) / dt + R(2) * k.vis_v;
    k.b_t = R(3) / dt + R(2) * k.vis_t;
    k.v_T = (R)h->params.v_T;
    k.t_phi = (R)h->params.t_phi;
    k.two_dx = R(2) * dx;
    k.two_dy = R(2) * dy;
    k.two_dz = R(2) * dz;
    k.three_dt = R(3) / dt;
    k.inv_two_h = R(1) / k.two_h;
    k.inv_two_dx = R(1) / k.two_dx;
    k.inv_two_dy = R(1) / k.two_dy;
    k.inv_two_dz = R(1) / k.two_dz;
    k.nv_in_temp = h->bv_synced ? 1 : 0;
    k.skip_tile_loads = h->fault == ADI_FAULT_SKIP_TILE_LOADS ? 1 : 0;
    k.tile_wait_tries = k.skip_tile_loads ? 16 : 1 << 17;
    return k;
}

cudaEvent_t take_event(adi_handle *h)
{
    if (!h->ev_free.empty()) {
        cudaEvent_t e = h->ev_free.back();
        h->ev_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

// Launches through `launch` (which returns a cudaError_t), counting it under the
// kernel class `cls` with `bytes` algorithmic HBM bytes, and bracketing it with
// an event pair when profiling is on.
template <class F>
cudaError_t timed(adi_handle *h, int cls, int64_t bytes, F launch)
{
    h->launches[cls]++;
    h->bytes[cls] += bytes;
    if (!h->prof_on) return launch();
    cudaEvent_t a = take_event(h), b = take_event(h);
    if (!a || !b) return cudaErrorMemoryAllocation;
    cudaEventRecord(a, h->stream);
    cudaError_t e = launch();
    cudaEventRecord(b, h->stream);
    h->ev_pending.push_back({cls, a, b});
    return e;
}

cudaError_t fold_profile(adi_handle *h)
{
    if (h->ev_pending.empty()) return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return e;
    for (auto &r : h->ev_pending) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) h->ms[r.cls] += t;
        h->ev_free.push_back(r.a);
        h->ev_free.push_back(r.b);
    }
    h->ev_pending.clear();
    return cudaSuccess;
}

void free_all(adi_handle *h)
{
    cudaFree(h->adj_mem);
    h->adj_mem = nullptr;
    h->adj_cap = 0;
    cudaFree(h->mask_mem);
    h->mask_mem = nullptr;
    h->mask_cap = 0;
    for (auto &r : h->ev_pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : h->ev_free) cudaEventDestroy(e);
    h->ev_pending.clear();
    h->ev_free.clear();
    cudaFree(h->d_code);
    for (int v = 0; v < 4; v++) cudaFree(h->d_nv[v]);
    for (int l = 0; l < 5; l++)
        for (int v = 0; v < 4; v++) cudaFree(h->d_L[l][v]);
    for (int d = 0; d < 3; d++) {
        cudaFree(h->d_line_lo[d]);
        cudaFree(h->d_line_hi[d]);
        cudaFree(h->d_segs[d]);
    }
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.exec);
    h->graphs.clear();
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    h->cap_stream = nullptr;
    if (h->io_used) cudaEventSynchronize(h->ev_io_down);   // a download may still be writing host memory
    if (h->io_up) cudaStreamDestroy(h->io_up);
    if (h->io_down) cudaStreamDestroy(h->io_down);
    for (cudaEvent_t e : {h->ev_io_up, h->ev_io_ready, h->ev_io_down})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->ev_io_piece)
        if (e) cudaEventDestroy(e);
    for (int v = 0; v < 4; v++) cudaFree(h->d_io[v]);
    h->io_up = h->io_down = nullptr;
    cudaFreeHost(h->h_pin);
    cudaFree(h->d_res);
    cudaFree(h->d_scratch);
    cudaFree(h->d_err);
    cudaFree(h->d_psum);
    cudaFree(h->d_pcnt);
    cudaFree(h->d_sum);
    cudaFree(h->d_cnt);
}

// The solver contract (the reference relies on it too: stencils read +-1 without
// bounds checks, TimeLayer3D.h:256-259,338-343).
std::string check_contract(const adi_handle *h, const uint8_t *t, const uint8_t *bv, const uint8_t *bt)
{
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const long long sx = (long long)ny * nz, sy = nz;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                long long id = i * sx + j * sy + k;
                bool frame = i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1;
                if (t[id] == NODE_IN) {
                    if (frame) return "NODE_IN cell on the outer frame";
                    if (t[id - sx] == NODE_OUT || t[id + sx] == NODE_OUT || t[id - sy] == NODE_OUT ||
                        t[id + sy] == NODE_OUT || t[id - 1] == NODE_OUT || t[id + 1] == NODE_OUT)
                        return "NODE_IN cell next to a NODE_OUT cell";
                } else if (!frame && (bv[id] == BC_FREE || bt[id] == BC_FREE)) {
                    if ((t[id - sx] == NODE_IN && t[id + sx] == NODE_IN) ||
                        (t[id - sy] == NODE_IN && t[id + sy] == NODE_IN) ||
                        (t[id - 1] == NODE_IN && t[id + 1] == NODE_IN))
                        return "BC_FREE cell shared by two segments of one line";
                }
            }
    return "";
}

int line_len(const adi_handle *h, int dir) { return dir == 0 ? h->nx : (dir == 1 ? h->ny : h->nz); }

bool shape_ok(const adi_handle *h, int dir, const FastShape &s)
{
    if (s.mode == 1) return dir == 2 && zwarp_supported(h->nz, s.K, (int)esize(h));
    if (s.mode == 2 || s.mode == 4)
        return dir < 2 && xytma_supported(dir, h->nx, h->ny, h->nz, s.K, s.mode == 2 ? 16 : 8, (int)esize(h));
    if (s.mode == 3) return dir < 2 && xypair_supported(dir, h->nx, h->ny, h->nz, s.K, (int)esize(h));
    if (s.mode == 5) return dir < 2 && xycp_supported(dir, h->nx, h->ny, h->nz, s.K, (int)esize(h));
    return s.mode == 0 && fast_shape_supported(dir, s, line_len(h, dir), (int)esize(h));
}

// Dispatch of the fast sweep to the kernel variant named by the shape.
template <typename R>
cudaError_t launch_fast(adi_handle *h, int dir, CLayer<R> cur, CLayer<R> tin, Layer<R> next, Layer<R> tout,
                        const SweepConst<R> &k, int merges, const FastShape &s)
{
    const DomainView<R> d = view<R>(h);
    if (s.mode == 1)
        return launch_sweep_zwarp<R>(d, h->d_line_lo[2], h->d_line_hi[2], cur, tin, next, tout, k, merges, s.K,
                                     h->stream);
    if (s.mode == 2 || s.mode == 4)
        return launch_sweep_xytma<R>(dir, d, h->d_line_lo[dir], cur, tin, next, tout, k, merges, s.K,
                                     s.mode == 2 ? 16 : 8, h->d_err, h->stream);
    if (s.mode == 5)
        return launch_sweep_xycp<R>(dir, d, cur, tin, next, tout, k, merges, s.K, h->d_err, h->stream);
    if (s.mode == 3) {
        if constexpr (std::is_same<R, float>::value)
            return launch_sweep_xypair(dir, d, h->d_line_lo[dir], cur, tin, next, tout, k, merges, s.K, h->d_err,
                                       h->stream);
        return cudaErrorInvalidConfiguration;
    }
    return launch_sweep_fast<R>(dir, d, h->d_line_lo[dir], h->d_line_hi[dir], cur, tin, next, tout, k, merges, s,
                                h->stream);
}

// One global iteration of TimeStep (AdiSolver3D.cpp:335-357): Z (cur -> next),
// Y (next -> half), X (half -> next), each num_local times, every sweep merging
// into the nonlinear layer; the last X sweep merges twice (the extra merge after
// X).  The two nonlinear buffers swap roles after every sweep.
// One sweep of direction dir from layer src into layer dst, reading the nonlinear
// layer ta and writing tb (the caller swaps them).
// tin: the layer read as the nonlinear layer (h->ta, or cur for the first sweep of
// a step whose start wrote the boundary values only).
template <typename R>
cudaError_t launch_sweep_once(adi_handle *h, int dir, int src, int dst, const SweepConst<R> &k, int merges,
                              int tin = -1)
{
    if (tin < 0) tin = h->ta;
    if (h->solver == ADI_SOLVER_FAST)
        return launch_fast<R>(h, dir, clayer<R>(h, src), clayer<R>(h, tin), layer<R>(h, dst), layer<R>(h, h->tb), k,
                              merges, h->shape[dir]);
    return launch_sweep_exact<R>(dir, view<R>(h), h->d_line_lo[dir], h->d_line_hi[dir], clayer<R>(h, src),
                                 clayer<R>(h, tin), layer<R>(h, dst), layer<R>(h, h->tb), (R *)h->d_scratch, k,
                                 merges, h->stream);
}

template <typename R>
Layer<R> layer_of(void *const *f)
{
    Layer<R> x;
    for (int v = 0; v < 4; v++) x.f[v] = (R *)f[v];
    return x;
}

template <typename R>
CLayer<R> clayer_of(void *const *f)
{
    CLayer<R> x;
    for (int v = 0; v < 4; v++) x.f[v] = (const R *)f[v];
    return x;
}

// One global iteration (Z, Y, X sweeps, num_local each).  With a tape (the
// adjoint's record of this iteration: per sweep k, slot k holds the nonlinear
// layer the sweep reads in fields 0-3 and the layer it writes in fields 4-7), the
// nonlinear layers live in the tape itself: sweep k reads slot k's layer and
// writes its merged nonlinear layer straight into slot k + 1's (the next sweep's
// input), except the step's last sweep (last_iteration), whose output nothing
// reads.  Slot 0 of a step is the step start's copy of cur; the other slots'
// off-NODE_IN cells, which no sweep writes, must hold what every nonlinear layer
// holds there (cur after the boundary update: node values, unchanged OUT cells),
// which adjoint_run copies in once.  The written layer is copied into the tape.
template <typename R>
adi_status enqueue_global_iteration(adi_handle *h, R dt, int num_local, void *const *tape = nullptr,
                                    bool last_iteration = true, bool first_reads_cur = false)
{
    const int order[3] = {2, 1, 0};
    const int src[3] = {h->cur, h->nxt, h->half};
    const int dst[3] = {h->nxt, h->half, h->nxt};
    for (int q = 0; q < 3; q++) {
        const int dir = order[q];
        const SweepConst<R> k = sweep_const<R>(h, dir, dt);
        // algorithmic bytes: IN rows read cur, temp and write next, temp (16
        // values); end rows write next (4 values)
        const int64_t bytes = (int64_t)sizeof(R) * (16 * h->num_in + 4 * (h->seg_nodes[dir] - h->num_in));
        const int cls = dir == 0 ? ADI_K_SWEEP_X : (dir == 1 ? ADI_K_SWEEP_Y : ADI_K_SWEEP_Z);
        for (int l = 0; l < num_local; l++) {
            const int merges = (dir == 0 && l == num_local - 1) ? 2 : 1;
            const size_t fb = (size_t)h->n * sizeof(R);
            if (!tape) {
                const int tin = first_reads_cur && q == 0 && l == 0 ? h->cur : h->ta;
                CK(timed(h, cls, bytes, [&] { return launch_sweep_once<R>(h, dir, src[q], dst[q], k, merges, tin); }));
            } else {
                const bool final_sweep = last_iteration && q == 2 && l == num_local - 1;
                const CLayer<R> tin = clayer_of<R>(tape);
                const Layer<R> tout = final_sweep ? layer<R>(h, h->tb) : layer_of<R>(tape + 8);
                CK(timed(h, cls, bytes, [&] {
                    if (h->solver == ADI_SOLVER_FAST)
                        return launch_fast<R>(h, dir, clayer<R>(h, src[q]), tin, layer<R>(h, dst[q]), tout, k,
                                              merges, h->shape[dir]);
                    return launch_sweep_exact<R>(dir, view<R>(h), h->d_line_lo[dir], h->d_line_hi[dir],
                                                 clayer<R>(h, src[q]), tin, layer<R>(h, dst[q]), tout,
                                                 (R *)h->d_scratch, k, merges, h->stream);
                }));
                CK(launch_copy_fields(4, h->d_L[dst[q]], tape + 4, fb, h->stream));   // the layer it wrote
                tape += 8;
            }
            std::swap(h->ta, h->tb);
        }
    }
    return ADI_OK;
}

std::vector<FastShape> shape_candidates(const adi_handle *h, int dir)
{
    std::vector<FastShape> out;
    const int len = line_len(h, dir);
    if (dir == 2)
        for (int K : {4, 5, 8, 12}) {
            FastShape s{K, 0, (len + K - 1) / K, 1};
            if (shape_ok(h, dir, s)) out.push_back(s);
        }
    else {
        for (int K : {4, 8}) {
            FastShape s{K, 32, len / K, 3};
            if (shape_ok(h, dir, s)) out.push_back(s);
        }
        for (int K : {4, 8, 16}) {
            FastShape s{K, 16, len / K, 2};
            if (shape_ok(h, dir, s)) out.push_back(s);
            FastShape s8{K, 8, len / K, 4};
            if (shape_ok(h, dir, s8)) out.push_back(s8);
        }
        for (int K : {4, 5}) {
            FastShape s{K, 8, (len + K - 1) / K, 5};
            if (shape_ok(h, dir, s)) out.push_back(s);
        }
    }
    for (int K : {4, 8, 12, 16})
        for (int NL : {1, 2, 4, 8, 16, 32}) {
            if (dir != 2 && NL < 8) continue;   // X/Y: lanes run along k, keep >= 32-byte runs
            FastShape s{K, NL, (len + K - 1) / K, 0};
            if (s.NL * s.P < 64) continue;
            if (shape_ok(h, dir, s)) out.push_back(s);
        }
    return out;
}

// Autotuner: times every candidate shape of the fast sweep on this domain and keeps
// the fastest per direction.  The timed launches read cur and write only layers
// that every step rewrites before reading (half and the nonlinear buffers).
template <typename R>
adi_status autotune(adi_handle *h, int reps)
{
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    for (int dir = 0; dir < 3; dir++) {
        const SweepConst<R> k = sweep_const<R>(h, dir, (R)1e-3);
        float best = 1e30f;
        FastShape best_s = h->shape[dir];
        for (const FastShape &s : shape_candidates(h, dir)) {
            auto go = [&] {
                return launch_fast<R>(h, dir, clayer<R>(h, h->cur), clayer<R>(h, h->ta), layer<R>(h, h->half),
                                      layer<R>(h, h->tb), k, 1, s);
            };
            // a tensor map the driver will not encode rules the candidate out before any launch
            const cudaError_t e0 = go();
            if (e0 == cudaErrorInvalidValue && (s.mode == 2 || s.mode == 3 || s.mode == 4)) continue;
            CK(e0);
            float tmin = 1e30f;
            for (int r = 0; r < reps; r++) {
                CK(cudaEventRecord(a, h->stream));
                CK(go());
                CK(cudaEventRecord(b, h->stream));
                CK(cudaEventSynchronize(b));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, a, b));
                tmin = ms < tmin ? ms : tmin;
            }
            if (tmin < best) { best = tmin; best_s = s; }
        }
        h->shape[dir] = best_s;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    h->tuned = true;
    return ADI_OK;
}

// Reads and clears the device error flag; ADI_ERR_TIMEOUT if a kernel's bounded
// wait gave up.
adi_status check_device_flag(adi_handle *h)
{
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (flag) {
        CK(cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
        return fail(h, ADI_ERR_TIMEOUT, "a sweep's bounded wait for its input tiles gave up");
    }
    return ADI_OK;
}

// Divergence error of layer l into the pinned results, with the device error flag
// (enqueue only).
template <typename R>
adi_status enqueue_div_error(adi_handle *h, int l)
{
    CK(timed(h, ADI_K_DIV_ERROR, (int64_t)h->n * (1 + 3 * (int64_t)sizeof(R)), [&] {
        return launch_div_error<R>(view<R>(h), clayer<R>(h, l), (R)h->dx, (R)h->dy, (R)h->dz, h->d_psum, h->d_pcnt,
                                   DIV_BLOCKS, h->d_sum, h->d_cnt, h->stream);
    }));
    CK(cudaMemcpyAsync(&h->h_pin->sum, h->d_sum, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&h->h_pin->cnt, h->d_cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&h->h_pin->err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    return ADI_OK;
}

// Waits for an enqueued divergence error and returns it through *out.
adi_status read_div_error(adi_handle *h, double *out)
{
    CK(cudaStreamSynchronize(h->stream));
    *out = h->h_pin->cnt ? h->h_pin->sum / (double)h->h_pin->cnt : 0.0;
    if (h->h_pin->err) {
        h->h_pin->err = 0;
        CK(cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
        return fail(h, ADI_ERR_TIMEOUT, "a sweep's bounded wait for its input tiles gave up");
    }
    return ADI_OK;
}

template <typename R>
adi_status div_error_of(adi_handle *h, int l, double *out)
{
    adi_status s = enqueue_div_error<R>(h, l);
    if (s != ADI_OK) return s;
    return read_div_error(h, out);
}

// Everything one fixed-iteration step puts on the stream: the step start (with
// the boundary update for adi_step), num_global global iterations, and the
// divergence error when requested.
template <typename R>
adi_status enqueue_step(adi_handle *h, R dt, int num_global, int num_local, int compute_error, bool update_bnd)
{
    if (update_bnd) {
        // cur gets the node values first, so the nonlinear layer the first sweep
        // reads (temp = cur) is cur itself: only BOUND / VALVE cells are written
        // (layer_ops.cu, step_begin_at, says why that keeps every value a sweep reads)
        CK(timed(h, ADI_K_STEP_BEGIN, (int64_t)h->n + 20 * (int64_t)sizeof(R) * (h->n - h->num_in), [&] {
            return launch_step_begin<R>(view<R>(h), layer<R>(h, h->cur), layer<R>(h, h->nxt), layer<R>(h, h->ta),
                                        layer<R>(h, h->tb), true, h->stream, true);
        }));
    } else {
        CK(timed(h, ADI_K_STEP_BEGIN, (int64_t)h->n * (1 + 8 * (int64_t)sizeof(R)), [&] {
            return launch_step_begin<R>(view<R>(h), layer<R>(h, h->cur), layer<R>(h, h->nxt), layer<R>(h, h->ta),
                                        layer<R>(h, h->tb), false, h->stream);
        }));
    }
    for (int it = 0; it < num_global; it++) {
        adi_status s = enqueue_global_iteration<R>(h, dt, num_local, nullptr, true, update_bnd && it == 0);
        if (s != ADI_OK) return s;
    }
    if (compute_error) return enqueue_div_error<R>(h, h->nxt);
    return ADI_OK;
}

// The host side of the end of TimeStep (AdiSolver3D.cpp:363-390): the divergence
// value when it was computed, the guard, the layer swap.
adi_status finish_step(adi_handle *h, int compute_error)
{
    if (compute_error) {
        adi_status s = read_div_error(h, &h->diff_error);
        if (s != ADI_OK) return s;
    }
    if (h->diff_error > 0.01) {
        char buf[128];
        snprintf(buf, sizeof buf, "divergence error %.8f above 0.01", h->diff_error);
        return fail(h, ADI_ERR_DIVERGENCE, buf);
    }
    std::swap(h->cur, h->nxt);
    h->bv_synced = false;   // the new state holds the sweeps' boundary values
    return ADI_OK;
}

void invalidate_graphs(adi_handle *h)
{
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.exec);
    h->graphs.clear();
}

// Replays (capturing on first use) the graph of one fixed-iteration step for the
// handle's current layer roles.  Captures on the handle's private stream, so the
// caller's stream may be the legacy default stream; the graph is launched on the
// caller's stream.  The launch counters advance by what the graph holds.
template <typename R>
adi_status step_graph(adi_handle *h, R dt, int num_global, int num_local, int compute_error, bool update_bnd)
{
    uint64_t key[4];
    double dd = (double)dt;
    memcpy(&key[0], &dd, sizeof dd);
    key[1] = (uint64_t)num_global | ((uint64_t)num_local << 20) | ((uint64_t)(compute_error != 0) << 40) |
             ((uint64_t)update_bnd << 41) | ((uint64_t)h->bv_synced << 42);
    key[2] = (uint64_t)h->cur | ((uint64_t)h->nxt << 4) | ((uint64_t)h->half << 8) | ((uint64_t)h->ta << 12) |
             ((uint64_t)h->tb << 16);
    key[3] = (uint64_t)h->stream;
    for (auto &g : h->graphs)
        if (!memcmp(g.key, key, sizeof key)) {
            CK(cudaGraphLaunch(g.exec, h->stream));
            h->ta = g.post_ta;
            h->tb = g.post_tb;
            for (int c = 0; c < ADI_K_NUM; c++) {
                h->launches[c] += g.launches[c];
                h->bytes[c] += g.bytes[c];
            }
            return ADI_OK;
        }
    adi_handle::GraphEntry ge;
    memcpy(ge.key, key, sizeof key);
    int64_t l0[ADI_K_NUM], b0[ADI_K_NUM];
    memcpy(l0, h->launches, sizeof l0);
    memcpy(b0, h->bytes, sizeof b0);
    const int ta0 = h->ta, tb0 = h->tb;
    const cudaStream_t user = h->stream;
    h->stream = h->cap_stream;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    adi_status st = e == cudaSuccess ? enqueue_step<R>(h, dt, num_global, num_local, compute_error, update_bnd)
                                     : fail(h, ADI_ERR_CUDA, "cudaStreamBeginCapture failed");
    if (e == cudaSuccess) {
        cudaError_t e2 = cudaStreamEndCapture(h->stream, &graph);
        if (st == ADI_OK && e2 != cudaSuccess)
            st = fail(h, ADI_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e2));
    }
    h->stream = user;
    if (st == ADI_OK) {
        e = cudaGraphInstantiate(&ge.exec, graph, 0);
        if (e != cudaSuccess) st = fail(h, ADI_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    if (graph) cudaGraphDestroy(graph);
    for (int c = 0; c < ADI_K_NUM; c++) {
        ge.launches[c] = h->launches[c] - l0[c];
        ge.bytes[c] = h->bytes[c] - b0[c];
    }
    ge.post_ta = h->ta;
    ge.post_tb = h->tb;
    if (st != ADI_OK) {
        // nothing ran: restore the bookkeeping the capture advanced
        memcpy(h->launches, l0, sizeof l0);
        memcpy(h->bytes, b0, sizeof b0);
        h->ta = ta0;
        h->tb = tb0;
        cudaGetLastError();
        return st;
    }
    if (h->graphs.size() >= 16) {
        cudaGraphExecDestroy(h->graphs.front().exec);
        h->graphs.erase(h->graphs.begin());
    }
    h->graphs.push_back(ge);
    // run it for this step
    h->ta = ta0;
    h->tb = tb0;
    memcpy(h->launches, l0, sizeof l0);
    memcpy(h->bytes, b0, sizeof b0);
    return step_graph<R>(h, dt, num_global, num_local, compute_error, update_bnd);
}

template <typename R>
adi_status time_step(adi_handle *h, double dt, int num_global, int num_local, int compute_error, bool update_bnd)
{
    const R dtr = (R)dt;
    if (update_bnd) h->bv_synced = true;   // step_begin applies the boundary values first
    adi_status s;
    if (h->graphs_on && !h->prof_on) s = step_graph<R>(h, dtr, num_global, num_local, compute_error, update_bnd);
    else s = enqueue_step<R>(h, dtr, num_global, num_local, compute_error, update_bnd);
    if (s != ADI_OK) return s;
    return finish_step(h, compute_error);
}

// Tolerance mode: global iterations until the residual max|x - t| / max|x| over
// NODE_IN cells (x the iteration's result, t the nonlinear layer its last sweep
// linearised about) is <= tol, at most max_global of them.  The host reads the
// residual after each iteration, so this path runs eagerly.
template <typename R>
adi_status time_step_tol(adi_handle *h, double dt, int max_global, int num_local, double tol, int compute_error,
                         bool update_bnd, int *iters_used, double *residual)
{
    const R dtr = (R)dt;
    if (update_bnd) h->bv_synced = true;
    CK(timed(h, ADI_K_STEP_BEGIN, (int64_t)h->n * (1 + 8 * (int64_t)sizeof(R)), [&] {
        return launch_step_begin<R>(view<R>(h), layer<R>(h, h->cur), layer<R>(h, h->nxt), layer<R>(h, h->ta),
                                    layer<R>(h, h->tb), update_bnd, h->stream);
    }));
    int it = 0;
    double r = NAN;
    while (it < max_global) {
        adi_status s = enqueue_global_iteration<R>(h, dtr, num_local);
        if (s != ADI_OK) return s;
        it++;
        // after the last X sweep the buffers swapped: tb holds the layer it read
        CK(cudaMemsetAsync(h->d_res, 0, 2 * sizeof(unsigned long long), h->stream));
        CK(timed(h, ADI_K_OTHER, (int64_t)h->num_in * 8 * (int64_t)sizeof(R), [&] {
            return launch_residual<R>(view<R>(h), clayer<R>(h, h->nxt), clayer<R>(h, h->tb), h->d_res, h->stream);
        }));
        CK(cudaMemcpyAsync(h->h_pin->res, h->d_res, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        double dm, xm;
        if (sizeof(R) == 4) {
            float a, b;
            const uint32_t ua = (uint32_t)h->h_pin->res[0], ub = (uint32_t)h->h_pin->res[1];
            memcpy(&a, &ua, 4);
            memcpy(&b, &ub, 4);
            dm = a;
            xm = b;
        } else {
            memcpy(&dm, &h->h_pin->res[0], 8);
            memcpy(&xm, &h->h_pin->res[1], 8);
        }
        r = xm > 0 ? dm / xm : dm;
        if (r <= tol) break;
    }
    if (iters_used) *iters_used = it;
    if (residual) *residual = r;
    if (compute_error) {
        adi_status s = enqueue_div_error<R>(h, h->nxt);
        if (s != ADI_OK) return s;
    }
    return finish_step(h, compute_error);
}

// ---------------------------------------------------------------------------
// Adjoint: dJ/d(node values) and dJ/d(initial state) of n_steps adi_step calls,
// J the kinetic energy in a box at the end.  Checkpoints the state every
// ckpt_every steps; each window is run backward from a tape (per sweep: the
// nonlinear layer read and the layer written), which the forward pass records
// for the last window and a recomputation from the window's checkpoint for the
// others.
// ---------------------------------------------------------------------------

// One device allocation carved into 256-byte aligned pieces (thousands of tape
// fields would otherwise cost a cudaMalloc each).  The allocation belongs to the
// handle and is reused by later calls whose workspace fits.
struct DevArena {
    char *base = nullptr;
    size_t cap = 0, used = 0;
    cudaError_t reserve(adi_handle *h, size_t bytes)
    {
        if (h->adj_cap < bytes) {
            cudaFree(h->adj_mem);
            h->adj_mem = nullptr;
            h->adj_cap = 0;
            const cudaError_t e = cudaMalloc((void **)&h->adj_mem, bytes);
            if (e != cudaSuccess) return e;
            h->adj_cap = bytes;
        }
        base = h->adj_mem;
        cap = h->adj_cap;
        return cudaSuccess;
    }
    void *get(size_t bytes, cudaError_t &e)
    {
        const size_t b = (bytes + 255) / 256 * 256;
        if (e != cudaSuccess) return nullptr;
        if (used + b > cap) { e = cudaErrorMemoryAllocation; return nullptr; }
        void *p = base + used;
        used += b;
        return p;
    }
};

template <typename R>
adi_status adjoint_run(adi_handle *h, double dt, int ng, int nl, int n_steps, int ck, const int lo[3], const int hi[3],
                       double *J, void *nv_grad, void *state_grad)
{
    const size_t fb = (size_t)h->n * sizeof(R);
    const int S = ng * nl * 3;
    const int nck = (n_steps + ck - 1) / ck;
    const int win = ck < n_steps ? ck : n_steps;
    const size_t fbr = (fb + 255) / 256 * 256;
    DevArena mem;
    cudaError_t e = mem.reserve(h, fbr * ((size_t)nck * 4 + 4 * 7 + 2 + (size_t)win * S * 8) + 256 * (DIV_BLOCKS + 16));
    auto layer4 = [&](void **out) {
        for (int v = 0; v < 4; v++) out[v] = mem.get(fb, e);
    };
    std::vector<void *> ckpt((size_t)nck * 4), fin(4), cb(4), nb(4), hb(4), tb(4), nvb(4), lamb(4);
    for (int c = 0; c < nck; c++) layer4(&ckpt[(size_t)c * 4]);
    layer4(fin.data()); layer4(nb.data());
    // the three adjoint layers every backward step starts from zero, as one block
    // (one memset per step)
    char *zblk = (char *)mem.get(12 * fbr, e);
    for (int v = 0; v < 4 && zblk; v++) {
        cb[v] = zblk + v * fbr;
        hb[v] = zblk + (4 + v) * fbr;
        tb[v] = zblk + (8 + v) * fbr;
    }
    layer4(nvb.data()); layer4(lamb.data());
    R *ga = (R *)mem.get(fb, e), *gbp = (R *)mem.get(fb, e);
    double *psum = (double *)mem.get(sizeof(double) * DIV_BLOCKS, e), *dJ = (double *)mem.get(sizeof(double), e);
    std::vector<void *> tape((size_t)win * S * 8);
    for (auto &p : tape) p = mem.get(fb, e);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(h, e == cudaErrorMemoryAllocation ? ADI_ERR_CAPACITY : ADI_ERR_CUDA,
                    "adjoint buffers: " + std::string(cudaGetErrorString(e)));
    }
    auto copy4 = [&](void *const *dst, void *const *src) -> adi_status {
        CK(launch_copy_fields(4, src, dst, fb, h->stream));
        return ADI_OK;
    };
    auto zero4 = [&](void *const *dst) -> adi_status {
        for (int v = 0; v < 4; v++) CK(cudaMemsetAsync(dst[v], 0, fb, h->stream));
        return ADI_OK;
    };
    adi_status st;
    const R dtr = (R)dt;
    // one step with its tape (the recomputation of a window does the same)
    auto taped_step = [&](int t, int t0) -> adi_status {
        h->bv_synced = true;
        void *const *tp = &tape[(size_t)(t - t0) * S * 8];
        // the step start writes its nonlinear layer (cur after the boundary update)
        // straight into the tape slot the first sweep reads
        CK(timed(h, ADI_K_STEP_BEGIN, (int64_t)h->n * (1 + 8 * (int64_t)sizeof(R)), [&] {
            return launch_step_begin<R>(view<R>(h), layer<R>(h, h->cur), layer<R>(h, h->nxt), layer_of<R>(tp),
                                        layer<R>(h, h->tb), true, h->stream);
        }));
        for (int it = 0; it < ng; it++) {
            const adi_status s2 = enqueue_global_iteration<R>(h, dtr, nl, tp + (size_t)it * nl * 3 * 8, it == ng - 1);
            if (s2 != ADI_OK) return s2;
        }
        std::swap(h->cur, h->nxt);
        h->bv_synced = false;
        return ADI_OK;
    };
    // The tape's nonlinear-layer slots hold, off NODE_IN, what every nonlinear layer
    // holds there: cur after the boundary update (node values on BOUND / VALVE,
    // OUT cells as they are), the same in every step of the run.  One step start
    // into the handle's temp layers gives it; the sweeps then write only NODE_IN.
    CK(launch_step_begin<R>(view<R>(h), layer<R>(h, h->cur), layer<R>(h, h->nxt), layer<R>(h, h->ta),
                            layer<R>(h, h->tb), true, h->stream));
    for (size_t q = 0; q < (size_t)win * S; q++)
        if ((st = copy4(&tape[q * 8], h->d_L[h->ta])) != ADI_OK) return st;
    // ---- forward, keeping checkpoints; the last window records its tape directly ----
    const int last_t0 = (nck - 1) * ck;
    for (int t = 0; t < n_steps; t++) {
        if (t % ck == 0 && (st = copy4(&ckpt[(size_t)(t / ck) * 4], h->d_L[h->cur])) != ADI_OK) return st;
        if (t >= last_t0) {
            if ((st = taped_step(t, last_t0)) != ADI_OK) return st;
            continue;
        }
        h->bv_synced = true;
        if (h->graphs_on && !h->prof_on) st = step_graph<R>(h, dtr, ng, nl, 0, true);
        else st = enqueue_step<R>(h, dtr, ng, nl, 0, true);
        if (st != ADI_OK) return st;
        std::swap(h->cur, h->nxt);
        h->bv_synced = false;
    }
    if ((st = copy4(fin.data(), h->d_L[h->cur])) != ADI_OK) return st;
    CK(launch_objective<R>(view<R>(h), clayer_of<R>(fin.data()), lo, hi, layer_of<R>(cb.data()), psum, DIV_BLOCKS, dJ,
                           h->stream));
    if ((st = zero4(nvb.data())) != ADI_OK) return st;
    const DomainView<R> dv = view<R>(h);
    // ---- backward, one checkpoint window at a time ----
    for (int w = nck - 1; w >= 0; w--) {
        const int t0 = w * ck, t1 = t0 + ck < n_steps ? t0 + ck : n_steps;
        if (w < nck - 1) {   // the last window's tape is the forward pass's
            if ((st = copy4(h->d_L[h->cur], &ckpt[(size_t)w * 4])) != ADI_OK) return st;
            for (int t = t0; t < t1; t++)
                if ((st = taped_step(t, t0)) != ADI_OK) return st;
        }
        for (int t = t1 - 1; t >= t0; t--) {
            void *const *tp = &tape[(size_t)(t - t0) * S * 8];
            if ((st = copy4(nb.data(), cb.data())) != ADI_OK) return st;
            CK(cudaMemsetAsync(zblk, 0, 12 * fbr, h->stream));   // cb, hb, tb
            int q = S - 1;
            for (int it = ng - 1; it >= 0; it--)
                for (int dir = 0; dir < 3; dir++) {
                    void *const *sb = dir == 2 ? cb.data() : (dir == 1 ? nb.data() : hb.data());
                    void *const *db = dir == 1 ? hb.data() : nb.data();
                    const SweepConst<R> k = sweep_const<R>(h, dir, dtr);
                    for (int l = nl - 1; l >= 0; l--, q--) {
                        const int merges = (dir == 0 && l == nl - 1) ? 2 : 1;
                        CK(timed(h, ADI_K_OTHER, 0, [&] {
                            return launch_adjoint_sweep<R>(dir, dv, h->d_line_lo[dir], h->d_line_hi[dir],
                                                           clayer_of<R>(tp + (size_t)q * 8),
                                                           clayer_of<R>(tp + (size_t)q * 8 + 4), layer_of<R>(sb),
                                                           layer_of<R>(db), layer_of<R>(tb.data()),
                                                           layer_of<R>(nvb.data()), ga, gbp, (R *)h->d_scratch, k,
                                                           merges, h->adjoint_K, layer_of<R>(lamb.data()),
                                                           h->stream);
                        }));
                    }
                }
            CK(launch_adjoint_step_start<R>(dv, layer_of<R>(cb.data()), layer_of<R>(nb.data()), layer_of<R>(tb.data()),
                                            layer_of<R>(nvb.data()), h->stream));
        }
    }
    if ((st = copy4(h->d_L[h->cur], fin.data())) != ADI_OK) return st;
    CK(cudaMemcpyAsync(J, dJ, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    for (int v = 0; v < 4; v++) {
        if (nv_grad)
            CK(cudaMemcpyAsync((char *)nv_grad + (size_t)v * fb, nvb[v], fb, cudaMemcpyDeviceToHost, h->stream));
        if (state_grad)
            CK(cudaMemcpyAsync((char *)state_grad + (size_t)v * fb, cb[v], fb, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return check_device_flag(h);
}

// Layer index of a role: 0 cur, 1 next, 2 half, 3 the nonlinear layer the next
// sweep reads, 4 the one it writes.
int role_layer(const adi_handle *h, int role)
{
    const int l[5] = {h->cur, h->nxt, h->half, h->ta, h->tb};
    return l[role];
}

adi_status check_ready(adi_handle *h)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (!h->mask_set) return fail(h, ADI_ERR_STATE, "adi_set_mask has not been called");
    if (!h->segs_built) return fail(h, ADI_ERR_STATE, "adi_build_segments has not been called");
    if (!h->contract_ok) return fail(h, ADI_ERR_BAD_ARG, "mask breaks the solver contract: " + h->contract_msg);
    return ADI_OK;
}

} // namespace

extern "C" {

const char *adi_version(void) { return kVersion; }

adi_status adi_fluid_params_normalized(double Re, double Pr, double lambda, adi_fluid_params *out)
{
    if (!out || Re == 0.0 || Pr == 0.0 || lambda == 0.0) return ADI_ERR_BAD_ARG;
    out->v_T = 1.0;
    out->v_vis = 1.0 / Re;
    out->t_vis = 1.0 / (Re * Pr);
    out->t_phi = (lambda - 1) / (lambda * Re);
    return ADI_OK;
}

adi_status adi_fluid_params_dimensional(double vis, double rho, double R, double k, double cv, adi_fluid_params *out)
{
    if (!out || rho == 0.0 || cv == 0.0) return ADI_ERR_BAD_ARG;
    out->v_T = R;
    out->v_vis = vis / rho;
    out->t_vis = k / (rho * cv);
    out->t_phi = vis / (rho * cv);
    return ADI_OK;
}

adi_status adi_create(const adi_grid_desc *g, const adi_fluid_params *p, adi_handle **out)
{
    if (!g || !p || !out) return ADI_ERR_BAD_ARG;
    *out = nullptr;
    if (g->dimx < 3 || g->dimy < 3 || g->dimz < 3) return ADI_ERR_BAD_ARG;
    if (g->precision != ADI_FP32 && g->precision != ADI_FP64) return ADI_ERR_BAD_ARG;
    if (!(g->dx > 0) || !(g->dy > 0) || !(g->dz > 0)) return ADI_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ADI_ERR_NO_DEVICE;
    adi_handle *h = new (std::nothrow) adi_handle();
    if (!h) return ADI_ERR_CAPACITY;
    cudaGetDevice(&h->device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess || prop.major < 10) {
        delete h;
        return ADI_ERR_NO_DEVICE;
    }
    h->prec = g->precision;
    h->nx = g->dimx; h->ny = g->dimy; h->nz = g->dimz;
    h->n = (long long)g->dimx * g->dimy * g->dimz;
    h->dx = g->dx; h->dy = g->dy; h->dz = g->dz;
    h->params = *p;
    for (int d = 0; d < 3; d++) {
        h->shape[d] = FastShape{4, d == 2 ? 2 : 8, (line_len(h, d) + 3) / 4, 0};
        if (!shape_ok(h, d, h->shape[d])) h->shape[d] = FastShape{16, 8, (line_len(h, d) + 15) / 16, 0};
    }
    const size_t fb = (size_t)h->n * esize(h);
    auto alloc = [&](void **ptr, size_t bytes) { return cudaMalloc(ptr, bytes); };
    cudaError_t e = alloc((void **)&h->d_code, h->n);
    for (int v = 0; v < 4 && e == cudaSuccess; v++) e = alloc(&h->d_nv[v], fb);
    for (int l = 0; l < 5 && e == cudaSuccess; l++)
        for (int v = 0; v < 4 && e == cudaSuccess; v++) e = alloc(&h->d_L[l][v], fb);
    for (int d = 0; d < 3 && e == cudaSuccess; d++) {
        LineGeom lg = line_geom(d, h->nx, h->ny, h->nz);
        e = alloc((void **)&h->d_line_lo[d], sizeof(int) * lg.nlines);
        if (e == cudaSuccess) e = alloc((void **)&h->d_line_hi[d], sizeof(int) * lg.nlines);
    }
    h->scratch_bytes = 6 * fb;
    if (e == cudaSuccess) e = alloc(&h->d_scratch, h->scratch_bytes);
    if (e == cudaSuccess) e = alloc((void **)&h->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = alloc((void **)&h->d_psum, sizeof(double) * DIV_BLOCKS);
    if (e == cudaSuccess) e = alloc((void **)&h->d_pcnt, sizeof(unsigned long long) * DIV_BLOCKS);
    if (e == cudaSuccess) e = alloc((void **)&h->d_sum, sizeof(double));
    if (e == cudaSuccess) e = alloc((void **)&h->d_cnt, sizeof(unsigned long long));
    if (e == cudaSuccess) e = alloc((void **)&h->d_res, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_pin, sizeof(adi_handle::Pinned));
    if (e == cudaSuccess) memset(h->h_pin, 0, sizeof(adi_handle::Pinned));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        for (int l = 0; l < 5 && e == cudaSuccess; l++)
            for (int v = 0; v < 4 && e == cudaSuccess; v++) e = cudaMemset(h->d_L[l][v], 0, fb);
    if (e != cudaSuccess) {
        free_all(h);
        delete h;
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? ADI_ERR_CAPACITY : ADI_ERR_CUDA;
    }
    *out = h;
    return ADI_OK;
}

adi_status adi_destroy(adi_handle *h)
{
    if (!h) return ADI_OK;
    cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return ADI_OK;
}

adi_status adi_set_stream(adi_handle *h, void *stream)
{
    if (!h) return ADI_ERR_BAD_ARG;
    h->stream = (cudaStream_t)stream;
    return ADI_OK;
}

adi_status adi_set_solver(adi_handle *h, int kind)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (kind != ADI_SOLVER_EXACT && kind != ADI_SOLVER_FAST) return fail(h, ADI_ERR_BAD_ARG, "unknown solver kind");
    h->solver = kind;
    invalidate_graphs(h);
    return ADI_OK;
}

adi_status adi_set_fault_injection(adi_handle *h, int what)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (what != ADI_FAULT_NONE && what != ADI_FAULT_SKIP_TILE_LOADS)
        return fail(h, ADI_ERR_BAD_ARG, "unknown fault-injection mode");
    h->fault = what;
    invalidate_graphs(h);
    return ADI_OK;
}

const char *adi_last_error_string(const adi_handle *h)
{
    if (!h) return "null handle";
    return h->err.c_str();
}

adi_status adi_set_mask(adi_handle *h, const uint8_t *type, const uint8_t *bc_vel, const uint8_t *bc_temp,
                        const double *vx, const double *vy, const double *vz, const double *T)
{
    if (!h || !type || !bc_vel || !bc_temp || !vx || !vy || !vz || !T) return ADI_ERR_BAD_ARG;
    const long long n = h->n;
    std::vector<uint8_t> code(n);
    long long nin = 0;
    for (long long i = 0; i < n; i++) {
        if (type[i] > NODE_VALVE || bc_vel[i] > BC_FREE || bc_temp[i] > BC_FREE)
            return fail(h, ADI_ERR_BAD_ARG, "node type or BC code out of range at index " + std::to_string(i));
        code[i] = (uint8_t)(type[i] | (bc_vel[i] == BC_FREE ? CODE_VEL_FREE : 0) |
                            (bc_temp[i] == BC_FREE ? CODE_TEMP_FREE : 0));
        nin += type[i] == NODE_IN;
    }
    h->contract_msg = check_contract(h, type, bc_vel, bc_temp);
    h->contract_ok = h->contract_msg.empty();
    h->num_in = nin;
    CK(cudaMemcpyAsync(h->d_code, code.data(), n, cudaMemcpyHostToDevice, h->stream));
    const double *src[4] = {vx, vy, vz, T};
    const size_t fb = (size_t)n * esize(h);
    if (h->prec == ADI_FP64) {
        for (int v = 0; v < 4; v++) {
            CK(cudaMemcpyAsync(h->d_nv[v], src[v], fb, cudaMemcpyHostToDevice, h->stream));
            CK(cudaMemcpyAsync(h->d_L[h->cur][v], src[v], fb, cudaMemcpyHostToDevice, h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
    } else {
        std::vector<float> tmp(n);
        for (int v = 0; v < 4; v++) {
            for (long long i = 0; i < n; i++) tmp[i] = (float)src[v][i];
            CK(cudaMemcpyAsync(h->d_nv[v], tmp.data(), fb, cudaMemcpyHostToDevice, h->stream));
            CK(cudaMemcpyAsync(h->d_L[h->cur][v], tmp.data(), fb, cudaMemcpyHostToDevice, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
    }
    h->mask_set = true;
    h->segs_built = false;
    invalidate_graphs(h);
    h->bv_synced = true;   // the initial state is the node values
    return ADI_OK;
}

namespace {

// Device scratch of one mask build or sampled layer read: pieces of the handle's
// workspace for these, which grows to the largest request and is kept (a call
// allocates nothing after the first one of its size).  Every user synchronises
// the stream before returning, so the next call may reuse the pieces.
struct HandleScratch {
    adi_handle *h;
    size_t used = 0;
    static size_t round(size_t b) { return (b + 255) / 256 * 256; }
    // bytes: the sizes of all pieces the build will take, in order
    cudaError_t reserve(std::initializer_list<size_t> bytes)
    {
        size_t total = 0;
        for (size_t b : bytes) total += round(b < 16 ? 16 : b);
        if (h->mask_cap < total) {
            cudaFree(h->mask_mem);
            h->mask_mem = nullptr;
            h->mask_cap = 0;
            const cudaError_t e = cudaMalloc((void **)&h->mask_mem, total);
            if (e != cudaSuccess) return e;
            h->mask_cap = total;
        }
        used = 0;
        return cudaSuccess;
    }
    cudaError_t get(void **out, size_t bytes)
    {
        const size_t b = round(bytes < 16 ? 16 : bytes);
        if (used + b > h->mask_cap) return cudaErrorMemoryAllocation;
        *out = h->mask_mem + used;
        used += b;
        return cudaSuccess;
    }
};

// What adi_set_mask derives on the host from a mask, for a mask a device builder
// wrote into d_code / d_nv (and the initial state into cur): the contract check
// (the same rules and the same first failing cell as check_contract) and the
// NODE_IN count, both computed on the device.
adi_status finish_device_mask(adi_handle *h, unsigned long long *d_census)
{
    CK(launch_mask_census(h->d_code, h->nx, h->ny, h->nz, d_census, h->stream));
    unsigned long long census[2];
    CK(cudaMemcpyAsync(census, d_census, sizeof census, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    static const char *const rules[4] = {"", "NODE_IN cell on the outer frame", "NODE_IN cell next to a NODE_OUT cell",
                                         "BC_FREE cell shared by two segments of one line"};
    h->contract_msg = census[0] == ~0ull ? std::string() : std::string(rules[census[0] & 3]);
    h->contract_ok = h->contract_msg.empty();
    h->num_in = (long long)census[1];
    h->mask_set = true;
    h->segs_built = false;
    invalidate_graphs(h);
    h->bv_synced = true;   // the initial state is the node values
    return ADI_OK;
}

// Status words of a builder: writes outside the grid, loops stopped at their bound.
adi_status mask_status(adi_handle *h, const int *d_status, const char *what)
{
    int st[2] = {0, 0};
    CK(cudaMemcpyAsync(st, d_status, sizeof st, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (st[1] > 0)
        return fail(h, ADI_ERR_BAD_ARG,
                    std::string(what) + ": " + std::to_string(st[1]) +
                        " scanline walks do not end in the reference's float arithmetic (a near-degenerate triangle)");
    if (st[0] > 0)
        return fail(h, ADI_ERR_BAD_ARG,
                    std::string(what) + ": " + std::to_string(st[0]) + " writes fall outside the node grid");
    return ADI_OK;
}

} // namespace

adi_status adi_mask_shape3d(adi_handle *h, const float *verts, int nverts, const int *tris, int ntris, double base_T,
                            int *fill_passes)
{
    if (!h || nverts < 0 || ntris < 0 || (nverts > 0 && !verts) || (ntris > 0 && !tris)) return ADI_ERR_BAD_ARG;
    for (long long q = 0; q < 3ll * ntris; q++)
        if (tris[q] < 0 || tris[q] >= nverts)
            return fail(h, ADI_ERR_BAD_ARG, "triangle " + std::to_string(q / 3) + " names a vertex out of range");
    const long long n = h->n;
    HandleScratch sc{h};
    uint8_t *types = nullptr;
    float *dv = nullptr;
    int *dt = nullptr, *st = nullptr;
    CK(sc.reserve({(size_t)n, sizeof(float) * 3 * (size_t)nverts, sizeof(int) * 3 * (size_t)ntris, sizeof(int) * 8}));
    CK(sc.get((void **)&types, n));
    CK(sc.get((void **)&dv, sizeof(float) * 3 * (size_t)nverts));
    CK(sc.get((void **)&dt, sizeof(int) * 3 * (size_t)ntris));
    CK(sc.get((void **)&st, sizeof(int) * 8));   // [0..1] status, [2] flood flag, [4..7] census
    CK(cudaMemsetAsync(st, 0, sizeof(int) * 8, h->stream));
    if (nverts > 0) CK(cudaMemcpyAsync(dv, verts, sizeof(float) * 3 * (size_t)nverts, cudaMemcpyHostToDevice, h->stream));
    if (ntris > 0) CK(cudaMemcpyAsync(dt, tris, sizeof(int) * 3 * (size_t)ntris, cudaMemcpyHostToDevice, h->stream));
    if (!h->mask_set) {
        // a grid that has had no mask: Grid3D::Init's nodes (v = 0, T = 0, no-slip)
        CK(cudaMemsetAsync(h->d_code, 0, n, h->stream));
        for (int v = 0; v < 4; v++) CK(cudaMemsetAsync(h->d_nv[v], 0, n * esize(h), h->stream));
    }
    int passes = 0;
    // every pass but the last turns at least one cell, so n + 1 passes always reach the fixed point
    CK(launch_mask_shape3d(types, h->nx, h->ny, h->nz, dv, nverts, dt, ntris, st, st + 2,
                           (int)std::min<long long>(n + 1, INT_MAX), &passes, h->stream));
    if (fill_passes) *fill_passes = passes;
    adi_status s = mask_status(h, st, "shape rasterisation");
    if (s != ADI_OK) return s;
    const float bt = (float)base_T;   // (FTYPE)baseT
    if (h->prec == ADI_FP64)
        CK(launch_mask_shape3d_install<double>(types, h->d_code, layer_of<double>(h->d_nv), layer<double>(h, h->cur), n,
                                               (double)bt, h->stream));
    else
        CK(launch_mask_shape3d_install<float>(types, h->d_code, layer_of<float>(h->d_nv), layer<float>(h, h->cur), n, bt,
                                              h->stream));
    return finish_device_mask(h, (unsigned long long *)(st + 4));
}

adi_status adi_mask_sea(adi_handle *h, const float *depth, int depth_nx, int depth_ny, float zmin, double base_T,
                        const float in_vel[3], double in_T)
{
    if (!h || !depth || !in_vel || depth_nx <= 0 || depth_ny <= 0) return ADI_ERR_BAD_ARG;
    const long long n = h->n;
    HandleScratch sc{h};
    uint8_t *snap = nullptr;
    float *dd = nullptr;
    int *st = nullptr;
    CK(sc.reserve({(size_t)n, sizeof(float) * (size_t)depth_nx * depth_ny, sizeof(int) * 8}));
    CK(sc.get((void **)&snap, n));
    CK(sc.get((void **)&dd, sizeof(float) * (size_t)depth_nx * depth_ny));
    CK(sc.get((void **)&st, sizeof(int) * 8));   // [0..1] status, [2] flood flag, [4..7] census
    CK(cudaMemsetAsync(st, 0, sizeof(int) * 8, h->stream));
    CK(cudaMemcpyAsync(dd, depth, sizeof(float) * (size_t)depth_nx * depth_ny, cudaMemcpyHostToDevice, h->stream));
    const float v3[3] = {in_vel[0], in_vel[1], in_vel[2]};
    if (h->prec == ADI_FP64)
        CK(launch_mask_sea<double>(h->d_code, snap, layer_of<double>(h->d_nv), layer<double>(h, h->cur), h->nx, h->ny,
                                   h->nz, dd, depth_nx, depth_ny, zmin, (float)base_T, v3, (float)in_T, st, h->stream));
    else
        CK(launch_mask_sea<float>(h->d_code, snap, layer_of<float>(h->d_nv), layer<float>(h, h->cur), h->nx, h->ny,
                                  h->nz, dd, depth_nx, depth_ny, zmin, (float)base_T, v3, (float)in_T, st, h->stream));
    adi_status s = mask_status(h, st, "sea mask");
    if (s != ADI_OK) return s;
    return finish_device_mask(h, (unsigned long long *)(st + 4));
}

adi_status adi_mask_extrude2d(adi_handle *h, const uint8_t *type2d, const float *vel2d, const float *T2d,
                              int active_nz, double depth_var, double base_T)
{
    if (!h || !type2d || !vel2d || !T2d) return ADI_ERR_BAD_ARG;
    if (active_nz < 2 || active_nz > h->nz) return fail(h, ADI_ERR_BAD_ARG, "active_nz must lie in [2, nz]");
    const long long cols = (long long)h->nx * h->ny;
    for (long long c = 0; c < cols; c++)
        if (type2d[c] > NODE_VALVE) return fail(h, ADI_ERR_BAD_ARG, "2D node type out of range");
    HandleScratch sc{h};
    uint8_t *t2 = nullptr;
    float *v2 = nullptr, *T2 = nullptr;
    int *st = nullptr;
    CK(sc.reserve({(size_t)cols, sizeof(float) * 2 * cols, sizeof(float) * cols, sizeof(int) * 8}));
    CK(sc.get((void **)&t2, cols));
    CK(sc.get((void **)&v2, sizeof(float) * 2 * cols));
    CK(sc.get((void **)&T2, sizeof(float) * cols));
    CK(sc.get((void **)&st, sizeof(int) * 8));   // [0..1] status, [2] flood flag, [4..7] census
    CK(cudaMemsetAsync(st, 0, sizeof(int) * 8, h->stream));
    CK(cudaMemcpyAsync(t2, type2d, cols, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(v2, vel2d, sizeof(float) * 2 * cols, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(T2, T2d, sizeof(float) * cols, cudaMemcpyHostToDevice, h->stream));
    if (h->prec == ADI_FP64)
        CK(launch_mask_extrude2d<double>(h->d_code, layer_of<double>(h->d_nv), layer<double>(h, h->cur), h->nx, h->ny,
                                         h->nz, t2, v2, T2, active_nz, depth_var, (float)base_T, st, h->stream));
    else
        CK(launch_mask_extrude2d<float>(h->d_code, layer_of<float>(h->d_nv), layer<float>(h, h->cur), h->nx, h->ny,
                                        h->nz, t2, v2, T2, active_nz, depth_var, (float)base_T, st, h->stream));
    adi_status s = mask_status(h, st, "2D extrusion");
    if (s != ADI_OK) return s;
    return finish_device_mask(h, (unsigned long long *)(st + 4));
}

adi_status adi_mask_shape2d(const float *segs, const uint8_t *seg_type, int nseg, int nx, int ny, double start_T,
                            void *cuda_stream, uint8_t *type2d, uint8_t *bc2d, float *vel2d, float *T2d)
{
    if (nseg < 0 || nx < 1 || ny < 1 || (nseg > 0 && (!segs || !seg_type)) || !type2d || !bc2d || !vel2d || !T2d)
        return ADI_ERR_BAD_ARG;
    for (int q = 0; q < nseg; q++)
        if (seg_type[q] != NODE_BOUND && seg_type[q] != NODE_VALVE) return ADI_ERR_BAD_ARG;
    adi_handle *h = nullptr;   // no handle: CK reports the status only
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const long long n = (long long)nx * ny;
    struct Bufs {
        void *p[8] = {};
        ~Bufs()
        {
            for (void *q : p) cudaFree(q);
        }
    } b;
    CK(cudaMalloc(&b.p[0], sizeof(float) * 8 * (size_t)(nseg > 0 ? nseg : 1)));
    CK(cudaMalloc(&b.p[1], (size_t)(nseg > 0 ? nseg : 1)));
    CK(cudaMalloc(&b.p[2], sizeof(unsigned long long) * n));
    CK(cudaMalloc(&b.p[3], n));
    CK(cudaMalloc(&b.p[4], sizeof(float) * 2 * n));
    CK(cudaMalloc(&b.p[5], sizeof(float) * n));
    CK(cudaMalloc(&b.p[6], n));
    CK(cudaMalloc(&b.p[7], sizeof(int) * 4));
    CK(cudaMemsetAsync(b.p[7], 0, sizeof(int) * 4, st));
    if (nseg > 0) {
        CK(cudaMemcpyAsync(b.p[0], segs, sizeof(float) * 8 * (size_t)nseg, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(b.p[1], seg_type, nseg, cudaMemcpyHostToDevice, st));
    }
    int passes = 0;
    int *status = (int *)b.p[7];
    CK(launch_mask_shape2d((const float *)b.p[0], (const uint8_t *)b.p[1], nseg, nx, ny, (float)start_T,
                           (unsigned long long *)b.p[2], (uint8_t *)b.p[3], (float *)b.p[4], (float *)b.p[5],
                           (uint8_t *)b.p[6], status, status + 2, (int)std::min<long long>(n + 1, INT_MAX), &passes,
                           st));
    int hs[2] = {0, 0};
    CK(cudaMemcpyAsync(hs, status, sizeof hs, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(type2d, b.p[3], n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(bc2d, b.p[6], n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(vel2d, b.p[4], sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(T2d, b.p[5], sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hs[0] > 0 || hs[1] > 0) return ADI_ERR_BAD_ARG;   // a segment leaves the grid or never ends
    return ADI_OK;
}

adi_status adi_get_mask(adi_handle *h, uint8_t *type, uint8_t *bc_vel, uint8_t *bc_temp, double *vx, double *vy,
                        double *vz, double *T)
{
    if (!h || !type || !bc_vel || !bc_temp || !vx || !vy || !vz || !T) return ADI_ERR_BAD_ARG;
    if (!h->mask_set) return fail(h, ADI_ERR_STATE, "the handle has no mask");
    const long long n = h->n;
    std::vector<uint8_t> code(n);
    CK(cudaMemcpyAsync(code.data(), h->d_code, n, cudaMemcpyDeviceToHost, h->stream));
    double *dst[4] = {vx, vy, vz, T};
    std::vector<float> tmp(h->prec == ADI_FP64 ? 0 : n);
    for (int v = 0; v < 4; v++) {
        if (h->prec == ADI_FP64) {
            CK(cudaMemcpyAsync(dst[v], h->d_nv[v], n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        } else {
            CK(cudaMemcpyAsync(tmp.data(), h->d_nv[v], n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            for (long long i = 0; i < n; i++) dst[v][i] = tmp[i];
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    for (long long i = 0; i < n; i++) {
        type[i] = code[i] & CODE_TYPE;
        bc_vel[i] = (code[i] & CODE_VEL_FREE) ? BC_FREE : BC_NOSLIP;
        bc_temp[i] = (code[i] & CODE_TEMP_FREE) ? BC_FREE : BC_NOSLIP;
    }
    return ADI_OK;
}

adi_status adi_build_segments(adi_handle *h, adi_seg_stats *stats)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (!h->mask_set) return fail(h, ADI_ERR_STATE, "adi_set_mask has not been called");
    invalidate_graphs(h);
    adi_seg_stats st;
    memset(&st, 0, sizeof st);
    st.num_in = h->num_in;
    for (int dir = 0; dir < 3; dir++) {
        LineGeom lg = line_geom(dir, h->nx, h->ny, h->nz);
        int *d_cnt = nullptr, *d_max = nullptr;
        long long *d_nodes = nullptr, *d_off = nullptr;
        CK(cudaMalloc(&d_cnt, sizeof(int) * lg.nlines));
        CK(cudaMalloc(&d_max, sizeof(int) * lg.nlines));
        CK(cudaMalloc(&d_nodes, sizeof(long long) * lg.nlines));
        CK(cudaMalloc(&d_off, sizeof(long long) * lg.nlines));
        CK(launch_segment_scan(dir, h->nx, h->ny, h->nz, h->d_code, d_cnt, h->d_line_lo[dir], h->d_line_hi[dir],
                               d_max, d_nodes, h->stream));
        std::vector<int> cnt(lg.nlines), mx(lg.nlines);
        std::vector<long long> nodes(lg.nlines), off(lg.nlines);
        CK(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * lg.nlines, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(mx.data(), d_max, sizeof(int) * lg.nlines, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(nodes.data(), d_nodes, sizeof(long long) * lg.nlines, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        long long total = 0, tnodes = 0;
        int maxlen = 0, maxper = 0;
        for (int l = 0; l < lg.nlines; l++) {
            off[l] = total;
            total += cnt[l];
            tnodes += nodes[l];
            maxlen = mx[l] > maxlen ? mx[l] : maxlen;
            maxper = cnt[l] > maxper ? cnt[l] : maxper;
        }
        st.num_segments[dir] = total;
        st.num_nodes[dir] = tnodes;
        h->seg_nodes[dir] = tnodes;
        st.max_size[dir] = maxlen;
        st.max_per_line[dir] = maxper;
        cudaFree(h->d_segs[dir]);
        h->d_segs[dir] = nullptr;
        h->nsegs[dir] = total;
        if (total > 0) {
            CK(cudaMalloc(&h->d_segs[dir], sizeof(int32_t) * 7 * total));
            CK(cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * lg.nlines, cudaMemcpyHostToDevice, h->stream));
            CK(launch_segment_write(dir, h->nx, h->ny, h->nz, h->d_code, d_off, h->d_segs[dir], h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
        cudaFree(d_cnt);
        cudaFree(d_max);
        cudaFree(d_nodes);
        cudaFree(d_off);
    }
    h->segs_built = true;
    if (stats) *stats = st;
    if (h->solver == ADI_SOLVER_FAST && !h->tuned) return adi_autotune(h, 3);
    return ADI_OK;
}

adi_status adi_autotune(adi_handle *h, int reps)
{
    if (!h || reps < 1) return ADI_ERR_BAD_ARG;
    if (!h->segs_built) return fail(h, ADI_ERR_STATE, "adi_build_segments has not been called");
    invalidate_graphs(h);
    if (h->prec == ADI_FP64) return autotune<double>(h, reps);
    return autotune<float>(h, reps);
}

adi_status adi_get_fast_shape(adi_handle *h, int dir, int *K, int *NL, int *P)
{
    if (!h || dir < 0 || dir > 2) return ADI_ERR_BAD_ARG;
    const FastShape s = h->shape[dir];
    if (K) *K = s.K;
    if (NL)
        *NL = s.mode == 1 ? 0
                          : (s.mode == 2 ? -16 : (s.mode == 3 ? -32 : (s.mode == 4 ? -8 : (s.mode == 5 ? -1 : s.NL))));
    if (P) *P = (line_len(h, dir) + s.K - 1) / s.K;
    return ADI_OK;
}

adi_status adi_set_fast_shape(adi_handle *h, int dir, int K, int NL)
{
    if (!h || dir < 0 || dir > 2 || K <= 0) return ADI_ERR_BAD_ARG;
    const int len = line_len(h, dir);
    if (NL < 0 && NL != -8 && NL != -16 && NL != -32 && NL != -1)
        return fail(h, ADI_ERR_BAD_ARG, "unsupported fast-sweep shape");
    const int mode = NL == 0 ? 1 : (NL == -16 ? 2 : (NL == -32 ? 3 : (NL == -8 ? 4 : (NL == -1 ? 5 : 0))));
    FastShape s{K, NL == -1 ? 8 : (NL < 0 ? -NL : NL), (len + K - 1) / K, mode};
    if (!shape_ok(h, dir, s)) return fail(h, ADI_ERR_BAD_ARG, "unsupported fast-sweep shape");
    h->shape[dir] = s;
    h->tuned = true;
    invalidate_graphs(h);
    return ADI_OK;
}

adi_status adi_get_segments(adi_handle *h, int dir, int32_t *out7, int64_t cap, int64_t *count)
{
    if (!h || dir < 0 || dir > 2) return ADI_ERR_BAD_ARG;
    if (!h->segs_built) return fail(h, ADI_ERR_STATE, "adi_build_segments has not been called");
    if (count) *count = h->nsegs[dir];
    if (!out7) return ADI_OK;
    if (cap < h->nsegs[dir]) return fail(h, ADI_ERR_CAPACITY, "segment buffer too small");
    if (h->nsegs[dir] > 0) {
        CK(cudaMemcpyAsync(out7, h->d_segs[dir], sizeof(int32_t) * 7 * h->nsegs[dir], cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return ADI_OK;
}

adi_status adi_update_boundaries(adi_handle *h)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (!h->mask_set) return fail(h, ADI_ERR_STATE, "adi_set_mask has not been called");
    CK(timed(h, ADI_K_OTHER, 0, [&] {
        if (h->prec == ADI_FP64) return launch_update_boundaries<double>(view<double>(h), layer<double>(h, h->cur), h->stream);
        return launch_update_boundaries<float>(view<float>(h), layer<float>(h, h->cur), h->stream);
    }));
    h->bv_synced = true;
    return ADI_OK;
}

static adi_status step_impl(adi_handle *h, double dt, int num_global, int num_local, int compute_error, bool bnd)
{
    adi_status s = check_ready(h);
    if (s != ADI_OK) return s;
    if (num_global < 1 || num_local < 1) return fail(h, ADI_ERR_BAD_ARG, "num_global and num_local must be >= 1");
    if (!(dt > 0) || !std::isfinite(dt)) return fail(h, ADI_ERR_BAD_ARG, "dt must be positive and finite");
    if (h->prec == ADI_FP64) return time_step<double>(h, dt, num_global, num_local, compute_error, bnd);
    return time_step<float>(h, dt, num_global, num_local, compute_error, bnd);
}

// ---- step phases (decompositions that exchange data between sweeps) ----

adi_status adi_phase_begin(adi_handle *h, int update_boundaries)
{
    adi_status s = check_ready(h);
    if (s != ADI_OK) return s;
    const bool ub = update_boundaries != 0;
    if (ub) h->bv_synced = true;   // step_begin applies the boundary values first
    if (h->prec == ADI_FP64)
        CK(launch_step_begin<double>(view<double>(h), layer<double>(h, h->cur), layer<double>(h, h->nxt),
                                     layer<double>(h, h->ta), layer<double>(h, h->tb), ub, h->stream));
    else
        CK(launch_step_begin<float>(view<float>(h), layer<float>(h, h->cur), layer<float>(h, h->nxt),
                                    layer<float>(h, h->ta), layer<float>(h, h->tb), ub, h->stream));
    h->launches[ADI_K_STEP_BEGIN]++;
    return ADI_OK;
}

adi_status adi_phase_sweep(adi_handle *h, int dir, double dt, int merges)
{
    adi_status s = check_ready(h);
    if (s != ADI_OK) return s;
    if (dir < 0 || dir > 2 || (merges != 1 && merges != 2)) return fail(h, ADI_ERR_BAD_ARG, "bad sweep phase");
    if (!(dt > 0) || !std::isfinite(dt)) return fail(h, ADI_ERR_BAD_ARG, "dt must be positive and finite");
    const int src = dir == 2 ? h->cur : (dir == 1 ? h->nxt : h->half);
    const int dst = dir == 2 ? h->nxt : (dir == 1 ? h->half : h->nxt);
    if (h->prec == ADI_FP64) CK(launch_sweep_once<double>(h, dir, src, dst, sweep_const<double>(h, dir, dt), merges));
    else CK(launch_sweep_once<float>(h, dir, src, dst, sweep_const<float>(h, dir, (float)dt), merges));
    h->launches[dir == 0 ? ADI_K_SWEEP_X : (dir == 1 ? ADI_K_SWEEP_Y : ADI_K_SWEEP_Z)]++;
    std::swap(h->ta, h->tb);
    return ADI_OK;
}

adi_status adi_phase_div_sum(adi_handle *h, int role, double *sum, uint64_t *count)
{
    if (!h || !sum || !count || role < 0 || role > 4) return ADI_ERR_BAD_ARG;
    adi_status s = check_ready(h);
    if (s != ADI_OK) return s;
    const int l = role_layer(h, role);
    s = h->prec == ADI_FP64 ? enqueue_div_error<double>(h, l) : enqueue_div_error<float>(h, l);
    if (s != ADI_OK) return s;
    double mean = 0.0;
    s = read_div_error(h, &mean);
    *sum = h->h_pin->sum;
    *count = h->h_pin->cnt;
    return s;
}

adi_status adi_phase_end(adi_handle *h)
{
    adi_status s = check_ready(h);
    if (s != ADI_OK) return s;
    std::swap(h->cur, h->nxt);
    h->bv_synced = false;   // the new state holds the sweeps' boundary values
    return ADI_OK;
}

adi_status adi_role_pointers(adi_handle *h, int role, void **out4)
{
    if (!h || !out4 || role < 0 || role > 4) return ADI_ERR_BAD_ARG;
    const int l = role_layer(h, role);
    for (int v = 0; v < 4; v++) out4[v] = h->d_L[l][v];
    return ADI_OK;
}

adi_status adi_time_step(adi_handle *h, double dt, int num_global, int num_local, int compute_error)
{
    return step_impl(h, dt, num_global, num_local, compute_error, false);
}

adi_status adi_step(adi_handle *h, double dt, int num_global, int num_local, int compute_error)
{
    return step_impl(h, dt, num_global, num_local, compute_error, true);
}

adi_status adi_run(adi_handle *h, double dt, int num_global, int num_local, int n_steps, int err_every)
{
    if (!h || n_steps < 0) return ADI_ERR_BAD_ARG;
    for (int i = 0; i < n_steps; i++) {
        int ce = (err_every > 0 && i % err_every == 0) || i == n_steps - 1;
        adi_status s = adi_step(h, dt, num_global, num_local, ce);
        if (s != ADI_OK) return s;
    }
    return ADI_OK;
}

adi_status adi_step_tol(adi_handle *h, double dt, int max_global, int num_local, double tol, int compute_error,
                        int *iters_used, double *residual)
{
    adi_status s = check_ready(h);
    if (s != ADI_OK) return s;
    if (max_global < 1 || num_local < 1) return fail(h, ADI_ERR_BAD_ARG, "max_global and num_local must be >= 1");
    if (!(dt > 0) || !std::isfinite(dt)) return fail(h, ADI_ERR_BAD_ARG, "dt must be positive and finite");
    if (!(tol >= 0)) return fail(h, ADI_ERR_BAD_ARG, "tol must be >= 0");
    if (h->prec == ADI_FP64)
        return time_step_tol<double>(h, dt, max_global, num_local, tol, compute_error, true, iters_used, residual);
    return time_step_tol<float>(h, dt, max_global, num_local, tol, compute_error, true, iters_used, residual);
}

adi_status adi_adjoint_run(adi_handle *h, double dt, int num_global, int num_local, int n_steps, int ckpt_every,
                           const int box_lo[3], const int box_hi[3], double *J, void *nv_grad, void *state_grad)
{
    adi_status s = check_ready(h);
    if (s != ADI_OK) return s;
    if (!J || !box_lo || !box_hi || n_steps < 1 || ckpt_every < 1 || num_global < 1 || num_local < 1)
        return fail(h, ADI_ERR_BAD_ARG, "adjoint: bad arguments");
    if (!(dt > 0) || !std::isfinite(dt)) return fail(h, ADI_ERR_BAD_ARG, "dt must be positive and finite");
    const int dims[3] = {h->nx, h->ny, h->nz};
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        lo[a] = box_lo[a] < 0 ? 0 : box_lo[a];
        hi[a] = box_hi[a] > dims[a] ? dims[a] : box_hi[a];
    }
    if (h->prec == ADI_FP64) return adjoint_run<double>(h, dt, num_global, num_local, n_steps, ckpt_every, lo, hi, J,
                                                        nv_grad, state_grad);
    return adjoint_run<float>(h, dt, num_global, num_local, n_steps, ckpt_every, lo, hi, J, nv_grad, state_grad);
}

adi_status adi_set_adjoint_chunk(adi_handle *h, int K)
{
    if (!h || (K != 0 && K != 4 && K != 8 && K != -4 && K != -8)) return ADI_ERR_BAD_ARG;
    h->adjoint_K = K;
    return ADI_OK;
}

adi_status adi_set_node_values(adi_handle *h, const double *vx, const double *vy, const double *vz, const double *T)
{
    if (!h || !vx || !vy || !vz || !T) return ADI_ERR_BAD_ARG;
    if (!h->mask_set) return fail(h, ADI_ERR_STATE, "adi_set_mask has not been called");
    const double *src[4] = {vx, vy, vz, T};
    const size_t fb = (size_t)h->n * esize(h);
    if (h->prec == ADI_FP64) {
        for (int v = 0; v < 4; v++) CK(cudaMemcpyAsync(h->d_nv[v], src[v], fb, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    } else {
        std::vector<float> tmp(h->n);
        for (int v = 0; v < 4; v++) {
            for (long long i = 0; i < h->n; i++) tmp[i] = (float)src[v][i];
            CK(cudaMemcpyAsync(h->d_nv[v], tmp.data(), fb, cudaMemcpyHostToDevice, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
    }
    h->bv_synced = false;
    return ADI_OK;
}

adi_status adi_set_graphs(adi_handle *h, int on)
{
    if (!h) return ADI_ERR_BAD_ARG;
    h->graphs_on = on != 0;
    if (!h->graphs_on) invalidate_graphs(h);
    return ADI_OK;
}

adi_status adi_get_state(adi_handle *h, int which, void *u, void *v, void *w, void *T)
{
    if (!h || !u || !v || !w || !T || (which != 0 && which != 1)) return ADI_ERR_BAD_ARG;
    const int l = which == 0 ? h->cur : h->nxt;
    void *dst[4] = {u, v, w, T};
    const size_t fb = (size_t)h->n * esize(h);
    for (int f = 0; f < 4; f++)
        CK(cudaMemcpyAsync(dst[f], h->d_L[l][f], fb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return check_device_flag(h);
}

adi_status adi_set_state(adi_handle *h, const void *u, const void *v, const void *w, const void *T)
{
    if (!h || !u || !v || !w || !T) return ADI_ERR_BAD_ARG;
    const void *src[4] = {u, v, w, T};
    const size_t fb = (size_t)h->n * esize(h);
    for (int f = 0; f < 4; f++)
        CK(cudaMemcpyAsync(h->d_L[h->cur][f], src[f], fb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->bv_synced = false;
    return ADI_OK;
}

adi_status adi_step_io(adi_handle *h, const void *const *in4, void *const *out4, double dt, int num_global,
                       int num_local, int compute_error)
{
    if (!h || !in4 || !out4) return ADI_ERR_BAD_ARG;
    for (int f = 0; f < 4; f++)
        if (!in4[f] || !out4[f]) return ADI_ERR_BAD_ARG;
    adi_status st = check_ready(h);
    if (st != ADI_OK) return st;
    const size_t fb = (size_t)h->n * esize(h);
    constexpr int NP = adi_handle::IO_PIECES;
    if (!h->io_up) {
        cudaError_t e = cudaStreamCreateWithFlags(&h->io_up, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->io_down, cudaStreamNonBlocking);
        for (cudaEvent_t *ev : {&h->ev_io_up, &h->ev_io_ready, &h->ev_io_down})
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
        for (cudaEvent_t &ev : h->ev_io_piece)
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        for (int v = 0; v < 4 && e == cudaSuccess; v++) e = cudaMalloc(&h->d_io[v], fb);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(h, ADI_ERR_CUDA, std::string("step_io buffers: ") + cudaGetErrorString(e));
        }
    }
    // pieces of a field: byte ranges [q*pb, min((q+1)*pb, fb))
    const size_t pb = ((fb + NP - 1) / NP + 255) / 256 * 256;
    auto range = [&](int q, size_t &o, size_t &len) {
        o = std::min(fb, (size_t)q * pb);
        len = std::min(fb, o + pb) - o;
    };
    // upload into cur: after everything queued on the handle's stream (the previous
    // step and its copy-out read cur), and each piece after the previous call's
    // download of the same piece (the host buffer may be that call's output)
    CK(cudaEventRecord(h->ev_io_ready, h->stream));   // everything queued on the handle so far
    CK(cudaStreamWaitEvent(h->io_up, h->ev_io_ready, 0));
    for (int f = 0; f < 4; f++)
        for (int q = 0; q < NP; q++) {
            size_t o, len;
            range(q, o, len);
            if (!len) continue;
            if (h->io_used) CK(cudaStreamWaitEvent(h->io_up, h->ev_io_piece[f * NP + q], 0));
            CK(cudaMemcpyAsync((char *)h->d_L[h->cur][f] + o, (const char *)in4[f] + o, len, cudaMemcpyHostToDevice,
                               h->io_up));
        }
    CK(cudaEventRecord(h->ev_io_up, h->io_up));
    CK(cudaStreamWaitEvent(h->stream, h->ev_io_up, 0));
    h->bv_synced = false;
    st = step_impl(h, dt, num_global, num_local, compute_error, true);
    if (st != ADI_OK) return st;
    // copy the result out of the layers (after the previous download has read the
    // copy), then download it piece by piece
    if (h->io_used) CK(cudaStreamWaitEvent(h->stream, h->ev_io_down, 0));
    CK(launch_copy_fields(4, h->d_L[h->cur], h->d_io, fb, h->stream));
    CK(cudaEventRecord(h->ev_io_ready, h->stream));
    CK(cudaStreamWaitEvent(h->io_down, h->ev_io_ready, 0));
    for (int f = 0; f < 4; f++)
        for (int q = 0; q < NP; q++) {
            size_t o, len;
            range(q, o, len);
            if (len) CK(cudaMemcpyAsync((char *)out4[f] + o, (const char *)h->d_io[f] + o, len,
                                        cudaMemcpyDeviceToHost, h->io_down));
            CK(cudaEventRecord(h->ev_io_piece[f * NP + q], h->io_down));
        }
    CK(cudaEventRecord(h->ev_io_down, h->io_down));
    h->io_used = true;
    return ADI_OK;
}

adi_status adi_io_wait(adi_handle *h)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (!h->io_used) return ADI_OK;
    // the handle's stream too, so work queued after this call (or an event a caller
    // records on it) follows the last download
    CK(cudaStreamWaitEvent(h->stream, h->ev_io_down, 0));
    CK(cudaEventSynchronize(h->ev_io_down));
    return check_device_flag(h);
}

adi_status adi_get_layer(adi_handle *h, int outdimx, int outdimy, int outdimz, void *vout, double *Tout)
{
    if (!h || !vout || !Tout || outdimx < 0 || outdimy < 0 || outdimz < 0) return ADI_ERR_BAD_ARG;
    if (!h->mask_set) return fail(h, ADI_ERR_STATE, "adi_set_mask has not been called");
    if (outdimx == 0) outdimx = h->nx;
    if (outdimy == 0) outdimy = h->ny;
    if (outdimz == 0) outdimz = h->nz;
    const int l = h->nxt;
    if (h->prec == ADI_FP64) CK(launch_fill_missing<double>(view<double>(h), layer<double>(h, l), h->stream));
    else CK(launch_fill_missing<float>(view<float>(h), layer<float>(h, l), h->stream));
    // point sampling on the device; only the sampled grid crosses to the host
    const long long m = (long long)outdimx * outdimy * outdimz;
    const size_t vb = (size_t)m * 3 * esize(h), tbytes = (size_t)m * sizeof(double);
    HandleScratch sc{h};
    void *dv = nullptr, *dt = nullptr;
    CK(sc.reserve({vb, tbytes}));
    CK(sc.get(&dv, vb));
    CK(sc.get(&dt, tbytes));
    if (h->prec == ADI_FP64)
        CK(launch_sample_layer<double>(clayer<double>(h, l), h->nx, h->ny, h->nz, outdimx, outdimy, outdimz,
                                       (double *)dv, (double *)dt, h->stream));
    else
        CK(launch_sample_layer<float>(clayer<float>(h, l), h->nx, h->ny, h->nz, outdimx, outdimy, outdimz, (float *)dv,
                                      (double *)dt, h->stream));
    CK(cudaMemcpyAsync(vout, dv, vb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(Tout, dt, tbytes, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ADI_OK;
}

adi_status adi_div_error(adi_handle *h, double *out)
{
    if (!h || !out) return ADI_ERR_BAD_ARG;
    if (!h->mask_set) return fail(h, ADI_ERR_STATE, "adi_set_mask has not been called");
    if (!h->contract_ok) return fail(h, ADI_ERR_BAD_ARG, "mask breaks the solver contract: " + h->contract_msg);
    if (h->prec == ADI_FP64) return div_error_of<double>(h, h->cur, out);
    return div_error_of<float>(h, h->cur, out);
}

adi_status adi_set_profiling(adi_handle *h, int on)
{
    if (!h) return ADI_ERR_BAD_ARG;
    h->prof_on = on != 0;
    return ADI_OK;
}

adi_status adi_get_profile(adi_handle *h, adi_profile *out, int reset)
{
    if (!h || !out) return ADI_ERR_BAD_ARG;
    CK(fold_profile(h));
    for (int c = 0; c < ADI_K_NUM; c++) {
        out->launches[c] = h->launches[c];
        out->ms[c] = h->ms[c];
        out->bytes[c] = h->bytes[c];
    }
    if (reset) {
        memset(h->launches, 0, sizeof h->launches);
        memset(h->ms, 0, sizeof h->ms);
        memset(h->bytes, 0, sizeof h->bytes);
    }
    return ADI_OK;
}

adi_status adi_device_pointers(adi_handle *h, void *out8[8])
{
    if (!h || !out8) return ADI_ERR_BAD_ARG;
    for (int f = 0; f < 4; f++) {
        out8[f] = h->d_L[h->cur][f];
        out8[4 + f] = h->d_L[h->nxt][f];
    }
    h->bv_synced = false;   // the caller may write the state through these
    return ADI_OK;
}

} // extern "C"

// ===========================================================================
// Batches: many independent domains stepped together, one persistent launch per
// sweep direction over every domain's lines, the whole step replayed as a graph.
// ===========================================================================

struct adi_batch {
    int prec = ADI_FP32;
    std::vector<adi_handle *> hs;
    cudaStream_t stream = nullptr, cap_stream = nullptr;
    void *d_doms = nullptr;                 // BatchDomain<R>[n]
    std::vector<unsigned char> host_doms;   // its host image
    int2 *d_items[3] = {};
    int nitems[3] = {0, 0, 0};
    int K[3] = {4, 4, 4};
    // schedule: ADI_BATCH_PERSISTENT (one multi-domain launch per sweep) or
    // ADI_BATCH_MEMBER_GRAPHS (every member's own step, members spread over
    // `branches` concurrent graph branches)
    int schedule = 0;
    int branches = 1;
    static constexpr int MAX_BRANCHES = 4;
    cudaStream_t br[MAX_BRANCHES] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[MAX_BRANCHES] = {};
    std::vector<std::vector<int>> branch_members;   // members per branch, largest first
    int grid[3] = {0, 0, 0};
    long long max_cells = 0;
    double dt_loaded = NAN;                 // dt the uploaded sweep constants are for
    double *d_psum = nullptr, *d_sum = nullptr;
    unsigned long long *d_pcnt = nullptr, *d_cnt = nullptr;
    double *h_sum = nullptr;                // pinned, n each
    unsigned long long *h_cnt = nullptr;
    std::vector<double> diff_error;
    bool graphs_on = true;
    struct GraphEntry {
        uint64_t key[5];
        cudaGraphExec_t exec;
        int post_ta, post_tb;
        int64_t launches;
    };
    std::vector<GraphEntry> graphs;
    int64_t launches = 0;
    std::string err;
};

namespace {

constexpr int BATCH_DIV_BLOCKS = 32;

adi_status bfail(adi_batch *b, adi_status s, const std::string &m)
{
    if (b) b->err = m;
    return s;
}

#define BCK(call)                                                                                      \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return bfail(b, ADI_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
    } while (0)

void batch_invalidate(adi_batch *b)
{
    for (auto &g : b->graphs) cudaGraphExecDestroy(g.exec);
    b->graphs.clear();
}

// Host image of every domain's BatchDomain and the per-direction work lists.
template <typename R>
adi_status batch_build(adi_batch *b)
{
    const int n = (int)b->hs.size();
    b->host_doms.assign(sizeof(BatchDomain<R>) * n, 0);
    BatchDomain<R> *bd = reinterpret_cast<BatchDomain<R> *>(b->host_doms.data());
    std::vector<std::pair<long long, int2>> items[3];
    b->max_cells = 0;
    for (int q = 0; q < n; q++) {
        adi_handle *h = b->hs[q];
        bd[q].d = view<R>(h);
        for (int l = 0; l < 5; l++)
            for (int v = 0; v < 4; v++) bd[q].L[l][v] = (R *)h->d_L[l][v];
        bd[q].dx = h->dx;
        bd[q].dy = h->dy;
        bd[q].dz = h->dz;
        bd[q].vec_ok = (h->nz % (16 / (int)sizeof(R))) == 0;
        b->max_cells = std::max(b->max_cells, h->n);
        for (int dir = 0; dir < 3; dir++) {
            bd[q].lo[dir] = h->d_line_lo[dir];
            bd[q].hi[dir] = h->d_line_hi[dir];
            const LineGeom g = line_geom(dir, h->nx, h->ny, h->nz);
            if (b->K[dir] < 0) {
                // X/Y tile kernel: items (domain, tile of 8 lines), lines up to 32 |K| rows
                if (g.len > 32 * -b->K[dir])
                    return bfail(b, ADI_ERR_CAPACITY, "a domain's lines are too long for the batched tile sweep");
                const int ntiles = (dir == 0 ? h->ny : h->nx) * ((h->nz + 7) / 8);
                for (int tl = 0; tl < ntiles; tl++) items[dir].push_back({0, make_int2(q, tl)});
                bd[q].P[dir] = 32;
                bd[q].NL[dir] = 8;
                continue;
            }
            const int P = (g.len + b->K[dir] - 1) / b->K[dir];
            if (P > 256) return bfail(b, ADI_ERR_CAPACITY, "a domain's lines are too long for the batched sweep");
            const int NL = std::max(1, 256 / P);
            bd[q].P[dir] = P;
            bd[q].NL[dir] = NL;
            for (int l0 = 0; l0 < g.nlines; l0 += NL)
                items[dir].push_back({(long long)P * b->K[dir] * NL, make_int2(q, l0)});
        }
    }
    for (int dir = 0; dir < 3; dir++) {
        // longest items first (LPT order over the persistent CTAs)
        std::stable_sort(items[dir].begin(), items[dir].end(),
                         [](const std::pair<long long, int2> &a, const std::pair<long long, int2> &c) {
                             return a.first > c.first;
                         });
        std::vector<int2> w(items[dir].size());
        for (size_t i = 0; i < w.size(); i++) w[i] = items[dir][i].second;
        cudaFree(b->d_items[dir]);
        b->d_items[dir] = nullptr;
        b->nitems[dir] = (int)w.size();
        if (!w.empty()) {
            BCK(cudaMalloc((void **)&b->d_items[dir], sizeof(int2) * w.size()));
            BCK(cudaMemcpy(b->d_items[dir], w.data(), sizeof(int2) * w.size(), cudaMemcpyHostToDevice));
        }
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        b->grid[dir] = std::max(1, std::min(b->nitems[dir], sms * (b->K[dir] == 4 ? 2 : 1)));   // generic kernel
    }
    if (!b->d_doms) BCK(cudaMalloc(&b->d_doms, b->host_doms.size()));
    b->dt_loaded = NAN;
    batch_invalidate(b);
    return ADI_OK;
}

// Sweep constants of every domain for dt, uploaded when dt changes.
template <typename R>
adi_status batch_load_dt(adi_batch *b, double dt)
{
    if (dt == b->dt_loaded) return ADI_OK;
    BatchDomain<R> *bd = reinterpret_cast<BatchDomain<R> *>(b->host_doms.data());
    for (size_t q = 0; q < b->hs.size(); q++) {
        b->hs[q]->bv_synced = true;   // the batched step always applies the boundary values first
        for (int dir = 0; dir < 3; dir++) bd[q].kc[dir] = sweep_const<R>(b->hs[q], dir, (R)dt);
    }
    BCK(cudaStreamSynchronize(b->stream));
    BCK(cudaMemcpy(b->d_doms, b->host_doms.data(), b->host_doms.size(), cudaMemcpyHostToDevice));
    b->dt_loaded = dt;
    batch_invalidate(b);
    return ADI_OK;
}

// One batched sweep: the X/Y tile kernel (K < 0: tiles of 8 lines copied
// element-wise, chunks of |K| rows) or the generic chunked kernel (K > 0).
template <typename R>
cudaError_t batch_sweep(adi_batch *b, int dir, int K, int src, int tin, int dst, int tout, int merges)
{
    const BatchDomain<R> *doms = (const BatchDomain<R> *)b->d_doms;
    if (K < 0)
        return launch_sweep_xy_batch<R>(dir, -K, doms, b->d_items[dir], b->nitems[dir], src, tin, dst, tout, merges,
                                        b->hs[0]->d_err, b->stream);
    return launch_sweep_fast_batch<R>(dir, K, doms, b->d_items[dir], b->nitems[dir], b->grid[dir], src, tin, dst, tout,
                                      merges, b->stream);
}

// Members over branches: longest processing time first by cells, each branch's
// members largest first.
void batch_assign_branches(adi_batch *b)
{
    const int n = (int)b->hs.size();
    std::vector<int> order(n);
    for (int q = 0; q < n; q++) order[q] = q;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->hs[x]->n > b->hs[y]->n; });
    b->branch_members.assign(b->branches, {});
    std::vector<long long> load(b->branches, 0);
    for (int q : order) {
        int w = 0;
        for (int v = 1; v < b->branches; v++)
            if (load[v] < load[w]) w = v;
        b->branch_members[w].push_back(q);
        load[w] += b->hs[q]->n;
    }
}

// One member's own step (what adi_step enqueues) on a branch stream, its
// nonlinear layers starting from the batch's roles (ta0, tb0); ta / tb receive
// the roles after it.  The batch counts the launches, not the member; per-launch
// profiling events stay out of batch graphs.
template <typename R>
adi_status enqueue_member_step(adi_batch *b, adi_handle *h, cudaStream_t stream, int num_global, int num_local,
                               int compute_error, int ta0, int tb0, int &ta, int &tb)
{
    const cudaStream_t own = h->stream;
    int64_t l0[ADI_K_NUM], b0[ADI_K_NUM];
    memcpy(l0, h->launches, sizeof l0);
    memcpy(b0, h->bytes, sizeof b0);
    const bool prof = h->prof_on;
    h->prof_on = false;
    h->stream = stream;
    h->ta = ta0;
    h->tb = tb0;
    h->bv_synced = true;
    const adi_status s = enqueue_step<R>(h, (R)b->dt_loaded, num_global, num_local, compute_error, true);
    h->stream = own;
    h->prof_on = prof;
    for (int c = 0; c < ADI_K_NUM; c++) b->launches += h->launches[c] - l0[c];
    memcpy(h->launches, l0, sizeof l0);
    memcpy(h->bytes, b0, sizeof b0);
    ta = h->ta;
    tb = h->tb;
    h->ta = ta0;
    h->tb = tb0;
    return s == ADI_OK ? ADI_OK : bfail(b, s, std::string("member step: ") + h->err);
}

// The member-graph schedule: every member's own step (its solver, kernels and
// shapes, as adi_step enqueues it) on one of `branches` streams forked from and
// joined back into the batch stream, so one member's launch tails and gaps
// overlap another member's sweeps.  Inside a capture the streams become parallel
// graph branches.
template <typename R>
adi_status batch_enqueue_members(adi_batch *b, int num_global, int num_local, int compute_error, int &ta, int &tb)
{
    BCK(cudaEventRecord(b->ev_fork, b->stream));
    const int ta0 = ta, tb0 = tb;
    for (int w = 0; w < b->branches; w++) {
        if (b->branch_members[w].empty()) continue;
        BCK(cudaStreamWaitEvent(b->br[w], b->ev_fork, 0));
        for (int q : b->branch_members[w]) {
            const adi_status s = enqueue_member_step<R>(b, b->hs[q], b->br[w], num_global, num_local, compute_error,
                                                        ta0, tb0, ta, tb);
            if (s != ADI_OK) return s;
        }
        BCK(cudaEventRecord(b->ev_join[w], b->br[w]));
        BCK(cudaStreamWaitEvent(b->stream, b->ev_join[w], 0));
    }
    return ADI_OK;
}

template <typename R>
adi_status batch_enqueue(adi_batch *b, int num_global, int num_local, int compute_error, int &ta, int &tb)
{
    if (b->schedule == ADI_BATCH_MEMBER_GRAPHS)
        return batch_enqueue_members<R>(b, num_global, num_local, compute_error, ta, tb);
    const adi_handle *h0 = b->hs[0];
    const int n = (int)b->hs.size();
    const BatchDomain<R> *doms = (const BatchDomain<R> *)b->d_doms;
    BCK(launch_step_begin_batch<R>(doms, n, b->max_cells, h0->cur, h0->nxt, ta, tb, true, b->stream));
    b->launches++;
    const int order[3] = {2, 1, 0};
    const int src[3] = {h0->cur, h0->nxt, h0->half};
    const int dst[3] = {h0->nxt, h0->half, h0->nxt};
    for (int it = 0; it < num_global; it++)
        for (int q = 0; q < 3; q++) {
            const int dir = order[q];
            for (int l = 0; l < num_local; l++) {
                const int merges = (dir == 0 && l == num_local - 1) ? 2 : 1;
                BCK(batch_sweep<R>(b, dir, b->K[dir], src[q], ta, dst[q], tb, merges));
                b->launches += b->nitems[dir] > 0;
                std::swap(ta, tb);
            }
        }
    if (compute_error) {
        BCK(launch_div_error_batch<R>(doms, n, h0->nxt, BATCH_DIV_BLOCKS, b->d_psum, b->d_pcnt, b->d_sum, b->d_cnt,
                                      b->stream));
        b->launches += 2;
        BCK(cudaMemcpyAsync(b->h_sum, b->d_sum, sizeof(double) * n, cudaMemcpyDeviceToHost, b->stream));
        BCK(cudaMemcpyAsync(b->h_cnt, b->d_cnt, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, b->stream));
    }
    return ADI_OK;
}

template <typename R>
adi_status batch_step(adi_batch *b, double dt, int num_global, int num_local, int compute_error)
{
    adi_status s = batch_load_dt<R>(b, dt);
    if (s != ADI_OK) return s;
    adi_handle *h0 = b->hs[0];
    int ta = h0->ta, tb = h0->tb;
    if (b->graphs_on) {
        uint64_t key[5] = {0, 0, 0, 0, 0};
        memcpy(&key[0], &dt, sizeof dt);
        key[1] = (uint64_t)num_global | ((uint64_t)num_local << 20) | ((uint64_t)(compute_error != 0) << 40);
        key[2] = (uint64_t)h0->cur | ((uint64_t)h0->nxt << 4) | ((uint64_t)h0->half << 8) | ((uint64_t)ta << 12) |
                 ((uint64_t)tb << 16);
        key[3] = (uint64_t)b->stream;
        key[4] = (uint64_t)b->schedule | ((uint64_t)b->branches << 8);
        adi_batch::GraphEntry *ge = nullptr;
        for (auto &g : b->graphs)
            if (!memcmp(g.key, key, sizeof key)) ge = &g;
        if (!ge) {
            adi_batch::GraphEntry e;
            memcpy(e.key, key, sizeof key);
            const cudaStream_t user = b->stream;
            const int64_t l0 = b->launches;
            b->stream = b->cap_stream;
            cudaGraph_t graph = nullptr;
            BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            int ta2 = ta, tb2 = tb;
            s = batch_enqueue<R>(b, num_global, num_local, compute_error, ta2, tb2);
            cudaError_t ec = cudaStreamEndCapture(b->stream, &graph);
            b->stream = user;
            if (s != ADI_OK) {
                b->launches = l0;
                if (graph) cudaGraphDestroy(graph);
                return s;
            }
            if (ec != cudaSuccess) return bfail(b, ADI_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ec));
            cudaError_t ei = cudaGraphInstantiate(&e.exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ei != cudaSuccess) return bfail(b, ADI_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ei));
            e.post_ta = ta2;
            e.post_tb = tb2;
            e.launches = b->launches - l0;
            b->launches = l0;
            if (b->graphs.size() >= 8) {
                cudaGraphExecDestroy(b->graphs.front().exec);
                b->graphs.erase(b->graphs.begin());
            }
            b->graphs.push_back(e);
            ge = &b->graphs.back();
        }
        BCK(cudaGraphLaunch(ge->exec, b->stream));
        b->launches += ge->launches;
        ta = ge->post_ta;
        tb = ge->post_tb;
    } else {
        s = batch_enqueue<R>(b, num_global, num_local, compute_error, ta, tb);
        if (s != ADI_OK) return s;
    }
    const int n = (int)b->hs.size();
    bool diverged = false;
    if (compute_error) {
        BCK(cudaStreamSynchronize(b->stream));
        for (int q = 0; q < n; q++) {
            if (b->schedule == ADI_BATCH_MEMBER_GRAPHS) {
                // each member's own divergence sum and wait flag (its enqueue_div_error)
                adi_handle *h = b->hs[q];
                b->diff_error[q] = h->h_pin->cnt ? h->h_pin->sum / (double)h->h_pin->cnt : 0.0;
                if (h->h_pin->err) {
                    h->h_pin->err = 0;
                    BCK(cudaMemsetAsync(h->d_err, 0, sizeof(int), b->stream));
                    return bfail(b, ADI_ERR_TIMEOUT, "a member sweep's bounded wait for its input tiles gave up");
                }
            } else {
                b->diff_error[q] = b->h_cnt[q] ? b->h_sum[q] / (double)b->h_cnt[q] : 0.0;
            }
        }
    }
    for (int q = 0; q < n; q++) diverged |= b->diff_error[q] > 0.01;
    for (int q = 0; q < n; q++) {
        adi_handle *h = b->hs[q];
        h->ta = ta;
        h->tb = tb;
        h->diff_error = b->diff_error[q];
        if (!diverged) {
            std::swap(h->cur, h->nxt);
            h->bv_synced = false;
        }
    }
    if (diverged) return bfail(b, ADI_ERR_DIVERGENCE, "a domain's divergence error is above 0.01; no domain advanced");
    return ADI_OK;
}

// A batch step with host buffers: every member's state uploaded from in[4 q + f],
// the step, the new state downloaded into out[4 q + f].  Member-graph schedule:
// each branch stream runs, member after member, the upload, the member's own step
// and the download, so one branch's copies overlap the other branches' sweeps
// (members are independent).  Persistent schedule: all uploads, the batch step,
// all downloads.  The next call's work waits for this call's (its uploads may read
// this call's downloads).
template <typename R>
adi_status batch_step_io(adi_batch *b, const void *const *in, void *const *out, double dt, int num_global,
                         int num_local, int compute_error)
{
    const int n = (int)b->hs.size();
    adi_handle *h0 = b->hs[0];
    if (b->schedule != ADI_BATCH_MEMBER_GRAPHS) {
        for (int q = 0; q < n; q++) {
            adi_handle *h = b->hs[q];
            const size_t fb = (size_t)h->n * sizeof(R);
            for (int f = 0; f < 4; f++)
                BCK(cudaMemcpyAsync(h->d_L[h->cur][f], in[4 * q + f], fb, cudaMemcpyHostToDevice, b->stream));
        }
        adi_status s = batch_step<R>(b, dt, num_global, num_local, compute_error);
        if (s != ADI_OK) return s;
        for (int q = 0; q < n; q++) {
            adi_handle *h = b->hs[q];
            const size_t fb = (size_t)h->n * sizeof(R);
            for (int f = 0; f < 4; f++)
                BCK(cudaMemcpyAsync(out[4 * q + f], h->d_L[h->cur][f], fb, cudaMemcpyDeviceToHost, b->stream));
        }
        return ADI_OK;
    }
    adi_status s = batch_load_dt<R>(b, dt);
    if (s != ADI_OK) return s;
    const int cur = h0->cur, nxt = h0->nxt, ta0 = h0->ta, tb0 = h0->tb;
    int ta = ta0, tb = tb0;
    BCK(cudaEventRecord(b->ev_fork, b->stream));
    for (int w = 0; w < b->branches; w++) {
        if (b->branch_members[w].empty()) continue;
        BCK(cudaStreamWaitEvent(b->br[w], b->ev_fork, 0));
        for (int q : b->branch_members[w]) {
            adi_handle *h = b->hs[q];
            const size_t fb = (size_t)h->n * sizeof(R);
            for (int f = 0; f < 4; f++)
                BCK(cudaMemcpyAsync(h->d_L[cur][f], in[4 * q + f], fb, cudaMemcpyHostToDevice, b->br[w]));
            const adi_status st = enqueue_member_step<R>(b, h, b->br[w], num_global, num_local, compute_error, ta0,
                                                         tb0, ta, tb);
            if (st != ADI_OK) return st;
            for (int f = 0; f < 4; f++)   // the new state: next until the roles swap below
                BCK(cudaMemcpyAsync(out[4 * q + f], h->d_L[nxt][f], fb, cudaMemcpyDeviceToHost, b->br[w]));
        }
        BCK(cudaEventRecord(b->ev_join[w], b->br[w]));
        BCK(cudaStreamWaitEvent(b->stream, b->ev_join[w], 0));
    }
    bool diverged = false;
    if (compute_error) {
        BCK(cudaStreamSynchronize(b->stream));
        for (int q = 0; q < n; q++) {
            adi_handle *h = b->hs[q];
            b->diff_error[q] = h->h_pin->cnt ? h->h_pin->sum / (double)h->h_pin->cnt : 0.0;
            if (h->h_pin->err) {
                h->h_pin->err = 0;
                BCK(cudaMemsetAsync(h->d_err, 0, sizeof(int), b->stream));
                return bfail(b, ADI_ERR_TIMEOUT, "a member sweep's bounded wait for its input tiles gave up");
            }
        }
    }
    for (int q = 0; q < n; q++) diverged |= b->diff_error[q] > 0.01;
    for (int q = 0; q < n; q++) {
        adi_handle *h = b->hs[q];
        h->ta = ta;
        h->tb = tb;
        h->diff_error = b->diff_error[q];
        if (!diverged) {
            std::swap(h->cur, h->nxt);
            h->bv_synced = false;
        }
    }
    if (diverged) return bfail(b, ADI_ERR_DIVERGENCE, "a domain's divergence error is above 0.01; no domain advanced");
    return ADI_OK;
}

// Mean time of one whole step with the current schedule and chunk lengths,
// replayed from a graph captured for it; the layer roles are left as they were
// (the step is not finished: cur keeps the state).
template <typename R>
adi_status batch_time_step(adi_batch *b, double dt, int num_global, int num_local, int reps, float *ms)
{
    adi_status s = batch_load_dt<R>(b, dt);
    if (s != ADI_OK) return s;
    const adi_handle *h0 = b->hs[0];
    int ta = h0->ta, tb = h0->tb;
    const cudaStream_t user = b->stream;
    const int64_t l0 = b->launches;
    b->stream = b->cap_stream;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    s = batch_enqueue<R>(b, num_global, num_local, 0, ta, tb);
    cudaError_t ec = cudaStreamEndCapture(b->stream, &graph);
    b->stream = user;
    b->launches = l0;
    if (s != ADI_OK || ec != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return s != ADI_OK ? s : bfail(b, ADI_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ec));
    }
    cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return bfail(b, ADI_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ei));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, b->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = cudaGraphLaunch(exec, b->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaGraphExecDestroy(exec);
    BCK(e);
    *ms = t / reps;
    return ADI_OK;
}

void batch_free(adi_batch *b)
{
    batch_invalidate(b);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    for (int w = 0; w < adi_batch::MAX_BRANCHES; w++) {
        if (b->br[w]) cudaStreamDestroy(b->br[w]);
        if (b->ev_join[w]) cudaEventDestroy(b->ev_join[w]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    cudaFree(b->d_doms);
    for (int d = 0; d < 3; d++) cudaFree(b->d_items[d]);
    cudaFree(b->d_psum);
    cudaFree(b->d_pcnt);
    cudaFree(b->d_sum);
    cudaFree(b->d_cnt);
    cudaFreeHost(b->h_sum);
    cudaFreeHost(b->h_cnt);
}

} // namespace

extern "C" {

adi_status adi_batch_create(adi_handle *const *handles, int n, adi_batch **out)
{
    if (!handles || n < 1 || !out) return ADI_ERR_BAD_ARG;
    *out = nullptr;
    adi_handle *h0 = handles[0];
    for (int q = 0; q < n; q++) {
        adi_handle *h = handles[q];
        if (!h) return ADI_ERR_BAD_ARG;
        adi_status s = check_ready(h);
        if (s != ADI_OK) return s;
        if (h->prec != h0->prec || h->device != h0->device)
            return fail(h, ADI_ERR_BAD_ARG, "batch members must share precision and device");
        if (h->cur != h0->cur || h->nxt != h0->nxt || h->half != h0->half || h->ta != h0->ta || h->tb != h0->tb)
            return fail(h, ADI_ERR_STATE, "batch members must have stepped in lock step (same layer roles)");
        for (int r = 0; r < q; r++)
            if (handles[r] == h) return fail(h, ADI_ERR_BAD_ARG, "a handle appears twice in the batch");
    }
    adi_batch *b = new (std::nothrow) adi_batch();
    if (!b) return ADI_ERR_CAPACITY;
    b->prec = h0->prec;
    b->hs.assign(handles, handles + n);
    b->stream = h0->stream;
    b->diff_error.assign(n, 0.0);
    for (int q = 0; q < n; q++) b->diff_error[q] = handles[q]->diff_error;
    cudaError_t e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    for (int w = 0; w < adi_batch::MAX_BRANCHES; w++) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->br[w], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[w], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    batch_assign_branches(b);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_psum, sizeof(double) * BATCH_DIV_BLOCKS * n);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_pcnt, sizeof(unsigned long long) * BATCH_DIV_BLOCKS * n);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_sum, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_cnt, sizeof(unsigned long long) * n);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&b->h_sum, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&b->h_cnt, sizeof(unsigned long long) * n);
    adi_status s = e == cudaSuccess ? ADI_OK : ADI_ERR_CUDA;
    if (s == ADI_OK) s = b->prec == ADI_FP64 ? batch_build<double>(b) : batch_build<float>(b);
    if (s != ADI_OK) {
        batch_free(b);
        delete b;
        cudaGetLastError();
        return s;
    }
    *out = b;
    return ADI_OK;
}

adi_status adi_batch_destroy(adi_batch *b)
{
    if (!b) return ADI_OK;
    cudaStreamSynchronize(b->stream);
    batch_free(b);
    delete b;
    return ADI_OK;
}

adi_status adi_batch_set_stream(adi_batch *b, void *stream)
{
    if (!b) return ADI_ERR_BAD_ARG;
    b->stream = (cudaStream_t)stream;
    for (auto *h : b->hs) h->stream = b->stream;
    return ADI_OK;
}

adi_status adi_batch_set_graphs(adi_batch *b, int on)
{
    if (!b) return ADI_ERR_BAD_ARG;
    b->graphs_on = on != 0;
    if (!b->graphs_on) batch_invalidate(b);
    return ADI_OK;
}

adi_status adi_batch_set_chunk(adi_batch *b, int dir, int K)
{
    if (!b || dir < 0 || dir > 2 || (K != 4 && K != 8 && !(dir < 2 && (K == -4 || K == -5)))) return ADI_ERR_BAD_ARG;
    const int old = b->K[dir];
    b->K[dir] = K;
    adi_status s = b->prec == ADI_FP64 ? batch_build<double>(b) : batch_build<float>(b);
    if (s != ADI_OK) {
        b->K[dir] = old;
        if (b->prec == ADI_FP64) batch_build<double>(b);
        else batch_build<float>(b);
    }
    return s;
}

adi_status adi_batch_get_chunk(adi_batch *b, int dir, int *K)
{
    if (!b || dir < 0 || dir > 2 || !K) return ADI_ERR_BAD_ARG;
    *K = b->K[dir];
    return ADI_OK;
}

adi_status adi_batch_step(adi_batch *b, double dt, int num_global, int num_local, int compute_error)
{
    if (!b) return ADI_ERR_BAD_ARG;
    if (num_global < 1 || num_local < 1) return bfail(b, ADI_ERR_BAD_ARG, "num_global and num_local must be >= 1");
    if (!(dt > 0) || !std::isfinite(dt)) return bfail(b, ADI_ERR_BAD_ARG, "dt must be positive and finite");
    const adi_handle *h0 = b->hs[0];
    for (auto *h : b->hs)
        if (h->cur != h0->cur || h->nxt != h0->nxt || h->ta != h0->ta || h->tb != h0->tb)
            return bfail(b, ADI_ERR_STATE, "a batch member was stepped on its own; step members only through the batch");
    if (b->prec == ADI_FP64) return batch_step<double>(b, dt, num_global, num_local, compute_error);
    return batch_step<float>(b, dt, num_global, num_local, compute_error);
}

adi_status adi_batch_step_io(adi_batch *b, const void *const *in, void *const *out, double dt, int num_global,
                             int num_local, int compute_error)
{
    if (!b || !in || !out) return ADI_ERR_BAD_ARG;
    if (num_global < 1 || num_local < 1) return bfail(b, ADI_ERR_BAD_ARG, "num_global and num_local must be >= 1");
    if (!(dt > 0) || !std::isfinite(dt)) return bfail(b, ADI_ERR_BAD_ARG, "dt must be positive and finite");
    for (size_t i = 0; i < 4 * b->hs.size(); i++)
        if (!in[i] || !out[i]) return ADI_ERR_BAD_ARG;
    const adi_handle *h0 = b->hs[0];
    for (auto *h : b->hs)
        if (h->cur != h0->cur || h->nxt != h0->nxt || h->ta != h0->ta || h->tb != h0->tb)
            return bfail(b, ADI_ERR_STATE, "a batch member was stepped on its own; step members only through the batch");
    if (b->prec == ADI_FP64) return batch_step_io<double>(b, in, out, dt, num_global, num_local, compute_error);
    return batch_step_io<float>(b, in, out, dt, num_global, num_local, compute_error);
}

adi_status adi_batch_io_wait(adi_batch *b)
{
    if (!b) return ADI_ERR_BAD_ARG;
    BCK(cudaStreamSynchronize(b->stream));
    return ADI_OK;
}

adi_status adi_batch_autotune(adi_batch *b, double dt, int reps)
{
    if (!b || reps < 1 || !(dt > 0)) return ADI_ERR_BAD_ARG;
    // times one sweep per direction and chunk length; the sweeps write half and the
    // nonlinear buffers only, which every step rewrites before reading
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    const adi_handle *h0 = b->hs[0];
    for (int dir = 0; dir < 3; dir++) {
        float best = 1e30f;
        int bestK = b->K[dir];
        for (int K : {4, 8, -4, -5}) {
            if (K < 0 && dir == 2) continue;
            b->K[dir] = K;
            adi_status s = b->prec == ADI_FP64 ? batch_build<double>(b) : batch_build<float>(b);
            if (s != ADI_OK) continue;
            s = b->prec == ADI_FP64 ? batch_load_dt<double>(b, dt) : batch_load_dt<float>(b, dt);
            if (s != ADI_OK) return s;
            float tmin = 1e30f;
            for (int r = 0; r < reps + 1; r++) {
                BCK(cudaEventRecord(e0, b->stream));
                cudaError_t e = b->prec == ADI_FP64
                    ? batch_sweep<double>(b, dir, K, h0->cur, h0->ta, h0->half, h0->tb, 1)
                    : batch_sweep<float>(b, dir, K, h0->cur, h0->ta, h0->half, h0->tb, 1);
                BCK(e);
                BCK(cudaEventRecord(e1, b->stream));
                BCK(cudaEventSynchronize(e1));
                float ms = 0;
                BCK(cudaEventElapsedTime(&ms, e0, e1));
                if (r > 0 && ms < tmin) tmin = ms;
            }
            if (tmin < best) { best = tmin; bestK = K; }
        }
        b->K[dir] = bestK;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    adi_status s = b->prec == ADI_FP64 ? batch_build<double>(b) : batch_build<float>(b);
    if (s != ADI_OK) return s;
    // the schedule: whole steps of every candidate
    const int n = (int)b->hs.size();
    float best = 1e30f;
    int best_sched = ADI_BATCH_PERSISTENT, best_br = 1;
    for (int c = 0; c <= adi_batch::MAX_BRANCHES; c++) {
        const int sched = c == 0 ? ADI_BATCH_PERSISTENT : ADI_BATCH_MEMBER_GRAPHS;
        const int brs = c == 0 ? 1 : c;
        if (brs > n) break;
        b->schedule = sched;
        b->branches = brs;
        batch_assign_branches(b);
        float ms = 0.f;
        s = b->prec == ADI_FP64 ? batch_time_step<double>(b, dt, 1, 2, reps, &ms)
                                : batch_time_step<float>(b, dt, 1, 2, reps, &ms);
        if (s != ADI_OK) return s;
        if (ms < best) { best = ms; best_sched = sched; best_br = brs; }
    }
    b->schedule = best_sched;
    b->branches = best_br;
    batch_assign_branches(b);
    batch_invalidate(b);
    return ADI_OK;
}

adi_status adi_batch_set_schedule(adi_batch *b, int schedule, int branches)
{
    if (!b || (schedule != ADI_BATCH_PERSISTENT && schedule != ADI_BATCH_MEMBER_GRAPHS) || branches < 1 ||
        branches > adi_batch::MAX_BRANCHES)
        return ADI_ERR_BAD_ARG;
    b->schedule = schedule;
    b->branches = branches;
    batch_assign_branches(b);
    batch_invalidate(b);
    return ADI_OK;
}

adi_status adi_batch_get_schedule(adi_batch *b, int *schedule, int *branches)
{
    if (!b || !schedule || !branches) return ADI_ERR_BAD_ARG;
    *schedule = b->schedule;
    *branches = b->branches;
    return ADI_OK;
}

adi_status adi_batch_time_step(adi_batch *b, double dt, int num_global, int num_local, int reps, float *ms_out)
{
    if (!b || reps < 1 || !(dt > 0) || num_global < 1 || num_local < 1 || !ms_out) return ADI_ERR_BAD_ARG;
    return b->prec == ADI_FP64 ? batch_time_step<double>(b, dt, num_global, num_local, reps, ms_out)
                               : batch_time_step<float>(b, dt, num_global, num_local, reps, ms_out);
}

adi_status adi_batch_time_sweeps(adi_batch *b, double dt, int reps, float *ms_out)
{
    if (!b || reps < 1 || !(dt > 0) || !ms_out) return ADI_ERR_BAD_ARG;
    adi_status s = b->prec == ADI_FP64 ? batch_load_dt<double>(b, dt) : batch_load_dt<float>(b, dt);
    if (s != ADI_OK) return s;
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    const adi_handle *h0 = b->hs[0];
    for (int dir = 0; dir < 3; dir++) {
        float sum = 0.f;
        for (int r = 0; r < reps + 1; r++) {
            BCK(cudaEventRecord(e0, b->stream));
            cudaError_t e = b->prec == ADI_FP64
                ? batch_sweep<double>(b, dir, b->K[dir], h0->cur, h0->ta, h0->half, h0->tb, 1)
                : batch_sweep<float>(b, dir, b->K[dir], h0->cur, h0->ta, h0->half, h0->tb, 1);
            BCK(e);
            BCK(cudaEventRecord(e1, b->stream));
            BCK(cudaEventSynchronize(e1));
            float ms = 0;
            BCK(cudaEventElapsedTime(&ms, e0, e1));
            if (r > 0) sum += ms;
        }
        ms_out[dir] = sum / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ADI_OK;
}

adi_status adi_batch_div_errors(adi_batch *b, double *out)
{
    if (!b || !out) return ADI_ERR_BAD_ARG;
    for (size_t q = 0; q < b->hs.size(); q++) out[q] = b->diff_error[q];
    return ADI_OK;
}

adi_status adi_batch_launches(adi_batch *b, int64_t *out)
{
    if (!b || !out) return ADI_ERR_BAD_ARG;
    *out = b->launches;
    return ADI_OK;
}

const char *adi_batch_last_error_string(const adi_batch *b)
{
    if (!b) return "null batch";
    return b->err.c_str();
}

} // extern "C"
