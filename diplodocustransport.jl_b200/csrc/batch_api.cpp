// Batched mixed-precision contexts (precision DTB_MIXED): many independent instances of one
// grid share the operators; each slot holds one instance with its own f, dt/dt0 and step count.
//
// Per batched step: for every gain group (gain blocks sharing an input pair) one tcgen05 GEMM
// of the stacked G rows (BF16 hi+lo, per-row power-of-two scale) against the batch of
// vec(f1 x f2), then one epilogue kernel over all (row, instance) pairs. The GEMM's plan
// (column tile, one SM or an SM pair per tile, K splits) is autotuned at commit per shape. Slots step while the
// device step counter is below their stop step, so requests of different lengths share one
// captured graph; a finished slot keeps its state until it is read and re-admitted.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "batch_internal.h"
#include "ctx.h"

namespace dtb {

struct MixedGroup {
    int in1 = 0, in2 = 0;
    int M = 0, N1 = 0, n2 = 0, n2p = 0, n_cb = 0;
    std::vector<std::pair<int, int>> members;  // (output species, first stacked row)
    unsigned char* gt = nullptr;  // G tiles [m_tiles][T][hi, lo][128 x 128 B], pre-swizzled
    float* row_scale = nullptr;
    float* partial = nullptr;
    int bn = 256, n_tiles = 1, m_tiles = 1, n_splits = 1, tiles_per_split = 1, Bpad = 256, splits_per_cb = 0;
    bool pair = false;  // the CTA-pair kernel (cta_group::2) runs this group
    double tuned_us = 0;  // autotuner: measured GEMM time of the chosen plan (0: not timed here)
    double flops = 0;  // 3 MMAs x 2 x M x K x Bcap
    double bytes = 0;  // hi + lo bytes of G
};

constexpr int kAdmitRing = 8;

struct MixedState {
    int Bcap = 0;   // slots in the state matrix: the requested capacity rounded up to 4 (row stride)
    int Buser = 0;  // slots the caller may use
    std::vector<MixedGroup> groups;
    float* F[2] = {nullptr, nullptr};
    float* C[2] = {nullptr, nullptr};
    int cur = 0;
    float* sig = nullptr;   // [ns][Bcap]
    float* isig = nullptr;  // [ns][Bcap]
    double* dt_scale = nullptr;
    long long* stop_step = nullptr;
    unsigned long long* min_ratio = nullptr;
    int* nonfinite = nullptr;
    unsigned long long* gstep = nullptr;
    int* active_hi = nullptr;  // device: 1 + the highest slot that still steps
    int last_active_hi = -1;
    long long host_step = 0;
    MixedRowOps ops{};
    cudaGraphExec_t graph = nullptr;
    // graphs[p][n]: n consecutive batched steps (1 <= n <= graph_steps) starting on state buffer p
    std::vector<cudaGraphExec_t> graphs[2];
    // host round trip of one step as one graph per state buffer (dtb_batch_run_io with
    // page-locked host arrays): upload and pack, the step, unpack and download, error flag
    struct IoGraph {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t x = nullptr;
        cudaGraphNode_t h2d = nullptr, d2h = nullptr;
        const void* src = nullptr;
        void* dst = nullptr;
    } io_graph[2];
    int graph_steps = 16;
    std::vector<long long> h_stop, h_start;
    float* pin_col = nullptr;  // [2][n_mom] staging of one slot's f and compensation (reads)
    // admission records: a ring of kAdmitRing pinned host records, their device copies and an
    // event per entry (an entry is rewritten only after its previous scatter has run)
    unsigned char* adm_pin = nullptr;
    unsigned char* adm_dev = nullptr;
    cudaEvent_t adm_ev[8] = {};
    int adm_next = 0;
    double* io_all = nullptr;  // device staging of the whole batch, f64 [Buser][n_mom]
    int* sp_off = nullptr;     // device species offsets
    double* mom_w = nullptr;   // device energy weights (n_mom)
    double* mom_out = nullptr; // device moments [Bcap][ns][2]
    bool profiling = false;
    double prof_ms = 0;
    long long prof_n = 0;
    std::vector<cudaEvent_t> ev;
    int prof_pending = 0;
};

}  // namespace dtb

namespace {

// BF16 bits of x rounded to nearest, ties to even (NaN kept a NaN).
uint16_t bf16_bits_rn(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
    return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}
double bf16_value(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
// 2^floor(log2(m)) for a finite m > 0, else 1: a row scale that brings the row's largest
// magnitude into [1, 2) without rounding anything
double pow2_scale(double m) { return (m > 0 && std::isfinite(m)) ? std::ldexp(1.0, std::ilogb(m)) : 1.0; }

// Operand rows for the batched epilogue: values v = x / scale(row) stored as BF16 hi = bf16(v)
// and lo = bf16(v - hi) (together about 16 significant bits), hi halves first, then the lo
// halves, in one device allocation.
int upload_hi_lo(dtb_ctx* c, const std::vector<double>& scaled, __nv_bfloat16** dst) {
    const size_t n = scaled.size();
    std::vector<uint16_t> h(2 * std::max<size_t>(1, n), 0);
    for (size_t k = 0; k < n; ++k) {
        const uint16_t hi = bf16_bits_rn((float)scaled[k]);
        h[k] = hi;
        h[n + k] = bf16_bits_rn((float)(scaled[k] - bf16_value(hi)));
    }
    DTB_TRY(c->alloc(dst, sizeof(uint16_t) * h.size()));
    DTB_CUDA(cudaMemcpyAsync(*dst, h.data(), sizeof(uint16_t) * h.size(), cudaMemcpyHostToDevice, c->stream));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    return DTB_OK;
}

}  // namespace

namespace {

unsigned long long ord_enc_host(double x) {
    unsigned long long u;
    std::memcpy(&u, &x, 8);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
double ord_dec_host(unsigned long long e) {
    unsigned long long u = (e >> 63) ? (e & 0x7FFFFFFFFFFFFFFFull) : ~e;
    double x;
    std::memcpy(&x, &u, 8);
    return x;
}

}  // namespace

// ---------------------------------------------------------------- gain GEMM plans
namespace {

// One way to run a group's gain GEMM: the kernel (one SM per tile, or an SM pair sharing a
// 256 x 256 MMA), the column tile width and the requested number of K splits.
struct GemmPlan {
    int pair = 0;
    int bn = 256;
    int splits = 1;
    double us = 0;  // measured time of one GEMM with this plan (0: not measured)
};

// Plans chosen so far in this process, by shape; a cache file (dtb_set_tune_cache) seeds it and
// records what the autotuner measures, one line per shape:
//   sm<SMs>:M<rows>:N1<n1>:n2<n2>:cols<columns>:cells<cells> <pair> <bn> <splits> <us>
std::mutex g_plan_mu;
std::map<std::string, GemmPlan> g_plans;
std::string g_plan_file;

std::string plan_key(const dtb_ctx* c, const MixedGroup& G, int Bcols) {
    char k[160];
    std::snprintf(k, sizeof(k), "sm%d:M%d:N1%d:n2%d:cols%d:cells%d", c->num_sms, G.M, G.N1, G.n2, Bcols,
                  (int)c->n_space);
    return k;
}

bool plan_valid(const MixedGroup& G, const GemmPlan& p, int max_pairs) {
    if (p.bn != 64 && p.bn != 128 && p.bn != 256) return false;
    if (p.splits < 1) return false;
    if (p.pair && (p.bn != 256 || G.m_tiles % 2 != 0 || max_pairs <= 0)) return false;
    return true;
}

// Tile counts and K splits of a plan. The splits are aligned to the 64-wide input-2 blocks
// when that keeps nearly every requested split: a split then never reloads its f2 block in
// mid-stream.
void apply_plan(MixedGroup& G, const GemmPlan& p, int Bcols) {
    G.pair = p.pair != 0;
    G.bn = p.bn;
    G.n_tiles = (Bcols + p.bn - 1) / p.bn;
    G.Bpad = G.n_tiles * p.bn;
    const int T = G.n_cb * G.N1;
    const int S = std::max(1, std::min(p.splits, T));
    G.tiles_per_split = (T + S - 1) / S;
    G.n_splits = (T + G.tiles_per_split - 1) / G.tiles_per_split;
    const int k_cb = S / G.n_cb;
    G.splits_per_cb = 0;
    if (k_cb >= 1 && k_cb <= G.N1 && (double)(k_cb * G.n_cb) >= 0.95 * S) {
        G.splits_per_cb = k_cb;
        G.n_splits = k_cb * G.n_cb;
    }
}

// Splits that fill the device once: one CTA per SM, or one pair per co-resident cluster.
// K splits that fill the device once, or a whole number of times (at most kMaxWaves) when one
// fill would leave a hi*hi accumulator more K tiles than its bound. A GEMM kernel spreads a
// split's hi*hi products over 512 / bn - 1 tensor-memory accumulators (one on SM pairs). Each is
// FP32 and its error grows with the number of MMAs it sums (measured: about 2e-5 relative after
// 3,328 K values in one accumulator; config 3 reached 3e-4 in its state after 5,000 steps with
// 20,736 K values per accumulator), so the bound keeps the gain term's error at a few 1e-6:
// 16 K tiles per accumulator on one SM, 32 on SM pairs (where a second fill would double the
// tensor-bound step's partial traffic).
constexpr int kMaxTilesPerAccSm = 16;
constexpr int kMaxTilesPerAccPair = 32;
constexpr int kMaxWaves = 4;
int fill_splits(const dtb_ctx* c, const MixedGroup& G, int pair, int bn, int Bcols, int max_pairs) {
    const int n_tiles = (Bcols + bn - 1) / bn;
    const double units = pair ? (double)(G.m_tiles / 2 * n_tiles) : (double)(G.m_tiles * n_tiles);
    const double cap = pair ? max_pairs : c->num_sms;  // CTAs (pairs) the device runs at once
    // rounded down: one CTA more than the device holds would run in a second wave on its own
    const int fill = std::max(1, (int)(cap / units));
    const int per_split = pair ? kMaxTilesPerAccPair : kMaxTilesPerAccSm * (512 / bn - 1);
    const int T = G.n_cb * G.N1;
    const int need = (T + per_split - 1) / per_split;
    const int waves = std::min(kMaxWaves, std::max(1, (need + fill - 1) / fill));
    if (waves == 1) return fill;
    // several waves: as many splits as whole waves hold (the last wave then runs nearly full)
    return std::max(fill * waves, (int)(waves * cap / units));
}

// Without timing: the widest tile the columns fill, on SM pairs when the rows pair up.
GemmPlan heuristic_plan(const dtb_ctx* c, const MixedGroup& G, int Bcols, int max_pairs) {
    GemmPlan p;
    p.bn = Bcols >= 192 ? 256 : (Bcols > 64 ? 128 : 64);
    p.pair = (p.bn == 256 && G.m_tiles % 2 == 0 && max_pairs > 0) ? 1 : 0;
    p.splits = fill_splits(c, G, p.pair, p.bn, Bcols, max_pairs);
    return p;
}

}  // namespace

GemmArgs gemm_args(const dtb_ctx* c, const MixedGroup& G, const float* Fin) {
    const MixedState* m = c->mixed;
    GemmArgs a;
    a.gt = G.gt;
    a.M = G.M;
    a.N1 = G.N1;
    a.n2 = G.n2;
    a.n_cb = G.n_cb;
    a.off1 = (int)c->off[G.in1];
    a.off2 = (int)c->off[G.in2];
    a.tiles_per_split = G.tiles_per_split;
    a.n_splits = G.n_splits;
    a.splits_per_cb = G.splits_per_cb;
    a.m_tiles = G.m_tiles;
    a.n_tiles = G.n_tiles;
    a.Bcap = m->Buser;
    a.Bst = m->Bcap;
    a.n_space = c->n_space;
    a.n_mom = (int)c->n_mom;
    a.Bpad = G.Bpad;
    a.F = Fin;
    a.isig1 = m->isig + (size_t)G.in1 * m->Bcap;
    a.isig2 = m->isig + (size_t)G.in2 * m->Bcap;
    a.partial = G.partial;
    a.err = c->err;
    a.active_hi = m->active_hi;
    // tensor-bound when the MMAs take longer than streaming G at the copy rate (ridge of about
    // 250 FLOP per byte on a B200): config 2's group (384 FLOP/B) is, config 3's (96) is not
    a.ring_after_x0 = G.flops > 250.0 * G.bytes ? 1 : 0;
    return a;
}

cudaError_t launch_group_gemm(const dtb_ctx* c, const MixedGroup& G, const float* Fin) {
    const GemmArgs a = gemm_args(c, G, Fin);
    return G.pair ? launch_gain_gemm_pair(a, c->stream) : launch_gain_gemm(G.bn, a, c->stream);
}

// Times each candidate plan of one group on the device (every column running, the state at its
// committed zeros: tensor-core time does not depend on the values) and returns the fastest.
int tune_group(dtb_ctx* c, MixedGroup& G, int Bcols, int max_pairs, GemmPlan* best) {
    MixedState* m = c->mixed;
    std::vector<GemmPlan> cands;
    for (int bn : {64, 128, 256}) {
        if (bn > 64 && bn / 2 >= Bcols) continue;  // half the tile or more would be padding
        GemmPlan p;
        p.bn = bn;
        p.splits = fill_splits(c, G, 0, bn, Bcols, max_pairs);
        cands.push_back(p);
        if (bn == 256 && G.m_tiles % 2 == 0 && max_pairs > 0) {
            p.pair = 1;
            p.splits = fill_splits(c, G, 1, bn, Bcols, max_pairs);
            cands.push_back(p);
        }
    }
    *best = heuristic_plan(c, G, Bcols, max_pairs);
    if (cands.size() < 2) return DTB_OK;
    size_t scratch = 0;
    for (const GemmPlan& p : cands) {
        apply_plan(G, p, Bcols);
        scratch = std::max(scratch, sizeof(float) * (size_t)G.n_splits * G.Bpad * G.M);
    }
    // the timing run's scratch partials and events, released on every way out
    struct Scratch {
        float* part = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        MixedGroup* G = nullptr;
        ~Scratch() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            if (part) cudaFree(part);
            if (G) G->partial = nullptr;
        }
    } sc;
    sc.G = &G;
    DTB_CUDA(cudaMalloc(&sc.part, scratch));
    DTB_CUDA(cudaEventCreate(&sc.e0));
    DTB_CUDA(cudaEventCreate(&sc.e1));
    float* const part = sc.part;
    const cudaEvent_t e0 = sc.e0, e1 = sc.e1;
    const int all = Bcols;
    DTB_CUDA(cudaMemcpyAsync(m->active_hi, &all, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    double best_ms = 1e30;
    int rc = DTB_OK;
    for (const GemmPlan& p : cands) {
        apply_plan(G, p, Bcols);
        G.partial = part;
        constexpr int kWarm = 2, kRep = 5;
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < kWarm && e == cudaSuccess; ++k) e = launch_group_gemm(c, G, m->F[0]);
        if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
        for (int k = 0; k < kRep && e == cudaSuccess; ++k) e = launch_group_gemm(c, G, m->F[0]);
        if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {  // a plan this device cannot launch is skipped
            cudaGetLastError();
            continue;
        }
        const double per = ms / kRep;
        if (per < best_ms) {
            best_ms = per;
            *best = p;
            best->us = per * 1e3;
        }
    }
    const int zero = 0;
    cudaError_t e = cudaMemcpyAsync(m->active_hi, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    int kerr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&kerr, c->err, sizeof(int), cudaMemcpyDeviceToHost);
    DTB_CUDA(e);
    if (kerr != 0) {
        set_error("gain GEMM autotuning: a bounded device wait gave up (code " + std::to_string(kerr) + ")");
        rc = DTB_ETIMEOUT;
    }
    return rc;
}

// Plan of every gain group: a plan already chosen for the shape in this process (or read from
// the cache file), else the autotuner's (or, with DTB_FLAG_NO_AUTOTUNE, the heuristic's).
int plan_gemms(dtb_ctx* c, int Bcols, int max_pairs) {
    MixedState* m = c->mixed;
    const bool tune = (c->opts.flags & DTB_FLAG_NO_AUTOTUNE) == 0;
    for (auto& G : m->groups) {
        GemmPlan p;
        bool have = false;
        const std::string key = plan_key(c, G, Bcols);
        // held across lookup, tuning and store: concurrent commits of one shape get one plan
        std::unique_lock<std::mutex> lk(g_plan_mu, std::defer_lock);
        if (tune) {
            lk.lock();
            auto it = g_plans.find(key);
            if (it != g_plans.end() && plan_valid(G, it->second, max_pairs)) {
                p = it->second;
                have = true;
            }
        }
        if (!have) {
            if (tune) {
                DTB_TRY(tune_group(c, G, Bcols, max_pairs, &p));
                g_plans[key] = p;
                if (!g_plan_file.empty()) {
                    if (FILE* f = std::fopen(g_plan_file.c_str(), "a")) {
                        std::fprintf(f, "%s %d %d %d %.3f\n", key.c_str(), p.pair, p.bn, p.splits, p.us);
                        std::fclose(f);
                    }
                }
            } else {
                p = heuristic_plan(c, G, Bcols, max_pairs);
            }
        }
        apply_plan(G, p, Bcols);
        G.tuned_us = p.us;
        DTB_TRY(c->alloc(&G.partial, sizeof(float) * (size_t)G.n_splits * G.Bpad * G.M));
    }
    return DTB_OK;
}

// Builds the device layouts of a DTB_MIXED context.
int commit_mixed(dtb_ctx* c) {
    DTB_CHECK(c->opts.batch >= 1, DTB_EINVAL, "batched context needs opts.batch >= 1");
    // the tensor-core GEMM streams dense blocks: a sparse M_Bin is densified per block
    for (auto& kv : c->sgains) {
        const int so = std::get<0>(kv.first), s1 = std::get<1>(kv.first), s2 = std::get<2>(kv.first);
        auto key = std::make_tuple(so, s1, s2);
        GainStage& g = c->gains[key];
        g.out = so;
        g.in1 = s1;
        g.in2 = s2;
        DTB_CHECK(g.dev_src.empty(), DTB_EINVAL, "a sparse M_Bin cannot be summed with a device-resident gain block");
        const int64_t n1 = c->sz[s1], n2 = c->sz[s2];
        if (g.host.empty()) g.host.assign((size_t)(c->sz[so] * n1 * n2), 0.0);
        const SparseGain& s = kv.second;
        for (size_t q = 0; q < s.v.size(); ++q) g.host[(size_t)(((int64_t)s.a[q] * n1 + s.b[q]) * n2 + s.c[q])] += s.v[q];
    }
    c->sgains.clear();
    auto* m = new MixedState();
    c->mixed = m;
    m->Buser = c->opts.batch;
    m->Bcap = (int)round_up(c->opts.batch, 4);
    if (c->opts.graph_steps > 0) m->graph_steps = (c->opts.graph_steps + 1) / 2 * 2;
    for (auto& gp : m->graphs) gp.assign((size_t)m->graph_steps + 1, nullptr);
    MixedRowOps& ops = m->ops;
    const int B = m->Bcap;
    const int n_mom = (int)c->n_mom;
    // a slot holds n_space cells of n_mom states: the state matrix has n_state rows, and the gain
    // GEMM takes every (cell, slot) pair as a column
    const int n_st = (int)c->n_state, nsp = c->n_space;
    const int Bcols = nsp * B;
    cudaStream_t s = c->stream;

    // ---------------- gain groups
    std::map<std::pair<int, int>, int> gidx;
    for (auto& kv : c->gains) {
        GainStage& g = kv.second;
        auto key = std::make_pair(g.in1, g.in2);
        if (!gidx.count(key)) {
            gidx[key] = (int)m->groups.size();
            MixedGroup G;
            G.in1 = g.in1;
            G.in2 = g.in2;
            G.N1 = (int)c->sz[g.in1];
            G.n2 = (int)c->sz[g.in2];
            G.n2p = (int)round_up(G.n2, kMmaK);
            G.n_cb = G.n2p / kMmaK;
            m->groups.push_back(G);
        }
        MixedGroup& G = m->groups[(size_t)gidx[key]];
        G.members.push_back({g.out, G.M});
        G.M += (int)c->sz[g.out];
    }
    DTB_CHECK(m->groups.size() <= 16, DTB_EINVAL, "at most 16 input pairs in a batched context");
    c->has_bin = !c->gains.empty() || !c->losses.empty();
    for (auto& kv : c->gains) {
        GainStage& g = kv.second;
        MixedGroup& G = m->groups[(size_t)gidx[{g.in1, g.in2}]];
        if (!G.gt) {
            // whole m tiles, rows past M stay zero
            const size_t bytes = (size_t)((G.M + kMmaM - 1) / kMmaM) * G.n_cb * G.N1 * kGTileBytes;
            DTB_TRY(c->alloc(&G.gt, bytes));
            DTB_CUDA(cudaMemsetAsync(G.gt, 0, bytes, s));
            DTB_TRY(c->alloc(&G.row_scale, sizeof(float) * G.M));
        }
        int roff = 0;
        for (auto& mb : G.members)
            if (mb.first == g.out) roff = mb.second;
        const int64_t no = c->sz[g.out];
        const size_t elems = (size_t)(no * G.N1 * G.n2);
        float* tmp = nullptr;
        const float* srcf = nullptr;
        if (!g.host.empty()) {
            DTB_CHECK(g.dev_src.empty(), DTB_EINVAL, "a gain block cannot mix host and device uploads");
            std::vector<float> h(elems);
            for (size_t k = 0; k < elems; ++k) h[k] = (float)g.host[k];
            DTB_CUDA(cudaMalloc(&tmp, sizeof(float) * elems));
            // stream-ordered with the conversion kernel below: a plain cudaMemcpy from pageable
            // memory may return before its DMA lands, unordered with this non-blocking stream
            DTB_CUDA(cudaMemcpyAsync(tmp, h.data(), sizeof(float) * elems, cudaMemcpyHostToDevice, s));
            srcf = tmp;
        } else {
            DTB_CHECK(g.dev_src.size() == 1, DTB_EINVAL, "a device-resident gain block must be uploaded once");
            if (g.dev_src[0].second == DTB_DTYPE_F32) {
                srcf = static_cast<const float*>(g.dev_src[0].first);
            } else {
                DTB_CUDA(cudaMalloc(&tmp, sizeof(float) * elems));
                cudaError_t ce = launch_pad_rows<double, float>(static_cast<const double*>(g.dev_src[0].first),
                                                                (long long)(no * G.N1), G.n2, tmp, G.n2, s);
                DTB_CUDA(ce);
                srcf = tmp;
            }
        }
        DTB_CUDA(launch_split_rows(srcf, no, roff, G.N1, G.n2, G.n_cb, G.gt, G.row_scale + roff, s));
        DTB_CUDA(cudaStreamSynchronize(s));
        if (tmp) cudaFree(tmp);
        g.host.clear();
        g.host.shrink_to_fit();
    }
    for (int b : {64, 128, 256}) DTB_CUDA(prepare_gain_gemm(b));
    DTB_CUDA(prepare_mixed_rows());
    int max_pairs = 0;
    if (prepare_gain_gemm_pair(&max_pairs) != cudaSuccess) {  // no cluster pairs: one-SM plans only
        cudaGetLastError();
        max_pairs = 0;
    }
    for (auto& G : m->groups) {
        G.m_tiles = (G.M + kMmaM - 1) / kMmaM;
        G.flops = 3.0 * 2.0 * G.M * (double)G.N1 * G.n2 * m->Buser * nsp;
        G.bytes = 4.0 * G.M * (double)G.N1 * G.n2;
    }
    // ---------------- gain lookup per species
    {
        int e = 0;
        for (int sp = 0; sp < c->ns; ++sp) {
            ops.gain_ptr[sp] = e;
            for (size_t gi = 0; gi < m->groups.size(); ++gi)
                for (auto& mb : m->groups[gi].members)
                    if (mb.first == sp) {
                        DTB_CHECK(e < 64, DTB_EINVAL, "too many gain blocks per species");
                        ops.gain_grp[e] = (int)gi;
                        ops.gain_roff[e] = mb.second;
                        ++e;
                    }
        }
        ops.gain_ptr[c->ns] = e;
    }
    // ---------------- loss, grouped by row species: BF16 hi + lo of the rows divided by a
    // power-of-two scale per momentum row (common to the row's loss blocks, so the products of
    // all its blocks share one accumulator)
    {
        std::vector<long long> doff;
        std::vector<int> ld, coff, ncols;
        std::vector<double> data;
        std::vector<double> rmax((size_t)n_mom, 0.0);
        for (auto& kv : c->losses) {
            const int sp = kv.first.first;
            const int64_t nr = c->sz[sp], nc = c->sz[kv.first.second];
            for (int64_t r = 0; r < nr; ++r)
                for (int64_t k = 0; k < nc; ++k)
                    rmax[(size_t)(c->off[sp] + r)] = std::max(rmax[(size_t)(c->off[sp] + r)],
                                                               std::fabs(kv.second[(size_t)(r * nc + k)]));
        }
        std::vector<double> rscale((size_t)n_mom);
        for (int64_t a = 0; a < n_mom; ++a) rscale[(size_t)a] = pow2_scale(rmax[(size_t)a]);
        for (int sp = 0; sp < c->ns; ++sp) {
            ops.loss_ptr[sp] = (int)doff.size();
            for (auto& kv : c->losses) {
                if (kv.first.first != sp) continue;
                const int oth = kv.first.second;
                const int64_t nr = c->sz[sp], nc = c->sz[oth], l = round_up(nc, 8);
                // rows padded with zeros to a multiple of 8 (16-byte rows for the epilogue's async copies)
                doff.push_back((long long)data.size());
                ld.push_back((int)l);
                coff.push_back((int)c->off[oth]);
                ncols.push_back((int)nc);
                const size_t base = data.size();
                data.resize(base + (size_t)(nr * l), 0.0);
                for (int64_t r = 0; r < nr; ++r)
                    for (int64_t k = 0; k < nc; ++k)
                        data[base + (size_t)(r * l + k)] = kv.second[(size_t)(r * nc + k)] / rscale[(size_t)(c->off[sp] + r)];
            }
        }
        ops.loss_ptr[c->ns] = (int)doff.size();
        long long* d_doff;
        int *d_ld, *d_coff, *d_nc;
        __nv_bfloat16* d_data;
        float* d_rs;
        DTB_TRY(copy_host_ints(c, &d_doff, doff));
        DTB_TRY(copy_host_ints(c, &d_ld, ld));
        DTB_TRY(copy_host_ints(c, &d_coff, coff));
        DTB_TRY(copy_host_ints(c, &d_nc, ncols));
        DTB_TRY(upload_hi_lo(c, data, &d_data));
        DTB_TRY(copy_host_vec(c, &d_rs, rscale));
        ops.loss_data_off = d_doff;
        ops.loss_ld = d_ld;
        ops.loss_col_off = d_coff;
        ops.loss_ncols = d_nc;
        ops.loss_data = d_data;
        ops.loss_lo = (long long)std::max<size_t>(1, data.size());
        ops.loss_rscale = d_rs;
    }
    // ---------------- emission pieces: BF16 hi + lo of the rows divided by a power-of-two scale
    // per state row (common to the pieces over that row), rows padded with zeros to a multiple of 8
    {
        c->has_emi = !c->emis.empty();
        std::vector<long long> doff;
        std::vector<int> ld, r0v, c0v, ncv;
        std::vector<std::vector<int>> rows((size_t)n_st);
        std::vector<double> data;
        std::vector<double> rmax((size_t)n_st, 0.0);
        for (const EmiPiece& e : c->emis)
            for (int64_t r = 0; r < e.nrows; ++r)
                for (int64_t k = 0; k < e.ncols; ++k)
                    rmax[(size_t)(e.row0 + r)] = std::max(rmax[(size_t)(e.row0 + r)], std::fabs(e.data[(size_t)(r * e.ncols + k)]));
        std::vector<double> rscale((size_t)n_st);
        for (int64_t a = 0; a < n_st; ++a) rscale[(size_t)a] = pow2_scale(rmax[(size_t)a]);
        for (size_t p = 0; p < c->emis.size(); ++p) {
            const EmiPiece& e = c->emis[p];
            const int64_t l = round_up(e.ncols, 8);
            doff.push_back((long long)data.size());
            ld.push_back((int)l);
            r0v.push_back((int)e.row0);
            c0v.push_back((int)e.col0);
            ncv.push_back((int)e.ncols);
            const size_t base = data.size();
            data.resize(base + (size_t)(e.nrows * l), 0.0);
            for (int64_t r = 0; r < e.nrows; ++r) {
                for (int64_t k = 0; k < e.ncols; ++k)
                    data[base + (size_t)(r * l + k)] = e.data[(size_t)(r * e.ncols + k)] / rscale[(size_t)(e.row0 + r)];
                rows[(size_t)(e.row0 + r)].push_back((int)p);
            }
        }
        __nv_bfloat16* d_data = nullptr;
        float* d_rs = nullptr;
        DTB_TRY(upload_hi_lo(c, data, &d_data));
        DTB_TRY(copy_host_vec(c, &d_rs, rscale));
        ops.emi_lo = (long long)std::max<size_t>(1, data.size());
        ops.emi_rscale = d_rs;
        std::vector<int> rptr((size_t)n_st + 1, 0), piece;
        for (int i = 0; i < n_st; ++i) {
            rptr[(size_t)i] = (int)piece.size();
            for (int p : rows[(size_t)i]) piece.push_back(p);
        }
        rptr[(size_t)n_st] = (int)piece.size();
        int *d_rptr, *d_piece, *d_ld, *d_r0, *d_c0, *d_nc;
        long long* d_doff;
        DTB_TRY(copy_host_ints(c, &d_rptr, rptr));
        DTB_TRY(copy_host_ints(c, &d_piece, piece));
        DTB_TRY(copy_host_ints(c, &d_doff, doff));
        DTB_TRY(copy_host_ints(c, &d_ld, ld));
        DTB_TRY(copy_host_ints(c, &d_r0, r0v));
        DTB_TRY(copy_host_ints(c, &d_c0, c0v));
        DTB_TRY(copy_host_ints(c, &d_nc, ncv));
        ops.emi_rptr = d_rptr;
        ops.emi_piece = d_piece;
        ops.emi_data_off = d_doff;
        ops.emi_ld = d_ld;
        ops.emi_row0 = d_r0;
        ops.emi_col0 = d_c0;
        ops.emi_ncols = d_nc;
        ops.emi_data = d_data;
    }
    // ---------------- flux: CSR with duplicates summed, banded ELL (FP32), padding column -1
    {
        std::vector<std::vector<std::pair<int64_t, double>>> rows((size_t)n_st);
        for (size_t p = 0; p < c->flux_r.size(); ++p) rows[(size_t)c->flux_r[p]].push_back({c->flux_c[p], c->flux_v[p]});
        int w = 0;
        for (auto& r : rows) {
            std::stable_sort(r.begin(), r.end(), [](auto& x, auto& y) { return x.first < y.first; });
            std::vector<std::pair<int64_t, double>> mm;
            for (auto& e : r) {
                if (!mm.empty() && mm.back().first == e.first)
                    mm.back().second += e.second;
                else
                    mm.push_back(e);
            }
            r.swap(mm);
            w = std::max<int>(w, (int)r.size());
        }
        w = std::max(w, 1);
        std::vector<double> val((size_t)n_st * w, 0.0);
        std::vector<int> col((size_t)n_st * w, -1);
        for (int i = 0; i < n_st; ++i)
            for (size_t k = 0; k < rows[(size_t)i].size(); ++k) {
                col[(size_t)i * w + k] = (int)rows[(size_t)i][k].first;
                val[(size_t)i * w + k] = rows[(size_t)i][k].second;
            }
        float* d_val;
        int* d_col;
        DTB_TRY(copy_host_vec(c, &d_val, val));
        DTB_TRY(copy_host_ints(c, &d_col, col));
        ops.ell_w = w;
        ops.ell_val = d_val;
        ops.ell_col = d_col;
    }
    // ---------------- vectors and state
    {
        std::vector<double> invAp(c->Ap.size());
        for (size_t i = 0; i < invAp.size(); ++i) invAp[i] = (double)(1.0f / (float)c->Ap[i]);
        float *d_inv, *d_inj;
        DTB_TRY(copy_host_vec(c, &d_inv, invAp));
        DTB_TRY(copy_host_vec(c, &d_inj, c->inj));
        ops.invAp = d_inv;
        ops.inj = d_inj;
        // per-cell Vol and BinM.Domain
        std::vector<double> vol(c->Vol.begin(), c->Vol.end());
        float* d_vol;
        DTB_TRY(copy_host_vec(c, &d_vol, vol));
        ops.vol_cell = d_vol;
        ops.bin_on = nullptr;
        if (c->has_bin_domain) {
            std::vector<unsigned char> on((size_t)nsp, 0);
            for (int64_t k : c->bin_domain)
                if (k >= 0 && k < nsp) on[(size_t)k] = 1;
            unsigned char* d_on;
            DTB_TRY(copy_host_ints(c, &d_on, on));
            ops.bin_on = d_on;
        }
    }
    const size_t nb = (size_t)n_st * B;
    for (int k = 0; k < 2; ++k) {
        DTB_TRY(c->alloc(&m->F[k], sizeof(float) * nb));
        DTB_TRY(c->alloc(&m->C[k], sizeof(float) * nb));
        DTB_CUDA(cudaMemsetAsync(m->F[k], 0, sizeof(float) * nb, s));
        DTB_CUDA(cudaMemsetAsync(m->C[k], 0, sizeof(float) * nb, s));
    }
    DTB_TRY(c->alloc(&m->sig, sizeof(float) * (size_t)c->ns * B));
    DTB_TRY(c->alloc(&m->isig, sizeof(float) * (size_t)c->ns * B));
    {
        std::vector<float> ones((size_t)c->ns * B, 1.0f);
        DTB_CUDA(cudaMemcpyAsync(m->sig, ones.data(), sizeof(float) * ones.size(), cudaMemcpyHostToDevice, s));
        DTB_CUDA(cudaMemcpyAsync(m->isig, ones.data(), sizeof(float) * ones.size(), cudaMemcpyHostToDevice, s));
        DTB_CUDA(cudaStreamSynchronize(s));
    }
    DTB_TRY(c->alloc(&m->dt_scale, sizeof(double) * B));
    DTB_TRY(c->alloc(&m->stop_step, sizeof(long long) * B));
    DTB_TRY(c->alloc(&m->min_ratio, sizeof(unsigned long long) * B));
    DTB_TRY(c->alloc(&m->nonfinite, sizeof(int) * B));
    DTB_TRY(c->alloc(&m->active_hi, sizeof(int)));
    DTB_CUDA(cudaMemsetAsync(m->active_hi, 0, sizeof(int), s));
    m->last_active_hi = 0;
    DTB_TRY(c->alloc(&m->gstep, sizeof(unsigned long long)));
    DTB_TRY(c->alloc(&c->err, sizeof(int)));
    DTB_CUDA(cudaMemsetAsync(m->dt_scale, 0, sizeof(double) * B, s));
    DTB_CUDA(cudaMemsetAsync(m->stop_step, 0, sizeof(long long) * B, s));
    DTB_CUDA(cudaMemsetAsync(m->nonfinite, 0, sizeof(int) * B, s));
    DTB_CUDA(cudaMemsetAsync(m->gstep, 0, sizeof(unsigned long long), s));
    DTB_CUDA(cudaMemsetAsync(c->err, 0, sizeof(int), s));
    {
        std::vector<unsigned long long> inf((size_t)B, ord_enc_host(INFINITY));
        DTB_CUDA(cudaMemcpyAsync(m->min_ratio, inf.data(), sizeof(unsigned long long) * B, cudaMemcpyHostToDevice, s));
        DTB_CUDA(cudaStreamSynchronize(s));
    }
    {
        std::vector<int> spo(c->off, c->off + c->ns + 1);
        DTB_TRY(copy_host_ints(c, &m->sp_off, spo));
        DTB_TRY(c->alloc(&m->mom_w, sizeof(double) * (size_t)n_mom));
        DTB_TRY(c->alloc(&m->mom_out, sizeof(double) * 2 * (size_t)c->ns * B * nsp));
    }
    DTB_CUDA(cudaMallocHost(&m->pin_col, sizeof(float) * 2 * (size_t)n_st));
    {
        const size_t rb = admit_record(n_st, c->ns).bytes;
        DTB_CUDA(cudaMallocHost(&m->adm_pin, rb * kAdmitRing));
        DTB_TRY(c->alloc(&m->adm_dev, rb * kAdmitRing));
        for (int k = 0; k < kAdmitRing; ++k) DTB_CUDA(cudaEventCreateWithFlags(&m->adm_ev[k], cudaEventDisableTiming));
    }
    DTB_CUDA(cudaMallocHost(&c->pin_err, sizeof(int)));
    m->h_stop.assign((size_t)B, 0);
    m->h_start.assign((size_t)B, 0);
    // ---------------- GEMM plan per group: tile width, kernel and K splits (autotuned)
    DTB_TRY(plan_gemms(c, Bcols, max_pairs));
    ops.n_mom = n_mom;
    ops.n_state = n_st;
    ops.n_space = nsp;
    ops.Bcap = B;
    ops.n_species = c->ns;
    for (int sp = 0; sp <= c->ns; ++sp) ops.sp_off[sp] = (int)c->off[sp];
    for (size_t gi = 0; gi < m->groups.size(); ++gi) {
        const MixedGroup& G = m->groups[gi];
        ops.grp_partial[gi] = G.partial;
        ops.grp_stride[gi] = (long long)G.Bpad * G.M;
        ops.grp_nsplit[gi] = G.n_splits;
        ops.grp_M[gi] = G.M;
        ops.grp_rscale[gi] = G.row_scale;
        ops.grp_sig1[gi] = m->sig + (size_t)G.in1 * B;
        ops.grp_sig2[gi] = m->sig + (size_t)G.in2 * B;
    }
    // tiles whose rows share one species and one list of emission pieces that cover all of
    // them take the shared-memory tile products
    {
        const int tr = mixed_rows_tile_rows();
        const int n_tiles_r = (n_st + tr - 1) / tr;
        std::vector<std::vector<int>> emi_rows((size_t)n_st);
        for (size_t p = 0; p < c->emis.size(); ++p)
            for (int64_t r = 0; r < c->emis[p].nrows; ++r) emi_rows[(size_t)(c->emis[p].row0 + r)].push_back((int)p);
        std::vector<unsigned char> fast((size_t)n_tiles_r, 1);
        for (int t = 0; t < n_tiles_r; ++t) {
            const int a0 = t * tr, a1 = std::min(n_st, a0 + tr);
            const int s0 = species_of(c, a0 % n_mom);
            if (a0 / n_mom != (a1 - 1) / n_mom) fast[(size_t)t] = 0;  // the tile lies in one cell
            for (int a = a0; a < a1; ++a)
                if (species_of(c, a % n_mom) != s0 || emi_rows[(size_t)a] != emi_rows[(size_t)a0]) fast[(size_t)t] = 0;
            // and whose K chunks fit the kernel's job list
            int64_t jobs = 0;
            for (auto& kv : c->losses)
                if (kv.first.first == s0) jobs += (c->sz[kv.first.second] + kRowsChunk - 1) / kRowsChunk;
            for (int p : emi_rows[(size_t)a0]) jobs += (c->emis[(size_t)p].ncols + kRowsChunk - 1) / kRowsChunk;
            if (jobs > kRowsMaxJobs) fast[(size_t)t] = 0;
        }
        unsigned char* d_fast;
        DTB_TRY(copy_host_ints(c, &d_fast, fast));
        ops.tile_fast = d_fast;
        // the fast tiles' product chunks, in the layout of the loss and emission data above:
        // the loss blocks of the tile's species, then the emission pieces of its rows
        std::vector<RowJob> jobs((size_t)n_tiles_r * kRowsMaxJobs);
        std::vector<int> njobs((size_t)n_tiles_r, 0);
        struct Opnd {
            const __nv_bfloat16* T;  // hi half of row 0 of the operand block, column 0
            int ld, col0, nc;
        };
        std::vector<std::vector<Opnd>> loss_of((size_t)c->ns);  // per species
        {
            long long off = 0;
            for (int sp = 0; sp < c->ns; ++sp)
                for (auto& kv : c->losses) {
                    if (kv.first.first != sp) continue;
                    const int64_t nr = c->sz[sp], nc = c->sz[kv.first.second], l = round_up(nc, 8);
                    loss_of[(size_t)sp].push_back({ops.loss_data + off, (int)l, (int)c->off[kv.first.second], (int)nc});
                    off += nr * l;
                }
        }
        std::vector<long long> emi_off(c->emis.size());
        {
            long long off = 0;
            for (size_t p = 0; p < c->emis.size(); ++p) {
                emi_off[p] = off;
                off += c->emis[p].nrows * round_up(c->emis[p].ncols, 8);
            }
        }
        for (int t = 0; t < n_tiles_r; ++t) {
            if (!fast[(size_t)t]) continue;
            const int a0 = t * tr, cell = a0 / n_mom, s0 = species_of(c, a0 % n_mom);
            // the tile's operands at its first row: loss blocks read the tile's cell, emission
            // pieces their global columns; a loss block and an emission piece over the same state
            // rows share jobs
            std::vector<Opnd> L, E;
            if (c->has_bin)
                for (const Opnd& o : loss_of[(size_t)s0])
                    L.push_back({o.T + (size_t)(a0 - cell * n_mom - c->off[s0]) * o.ld, o.ld, o.col0 + cell * n_mom, o.nc});
            for (int p : emi_rows[(size_t)a0]) {
                const EmiPiece& e = c->emis[(size_t)p];
                const int l = (int)round_up(e.ncols, 8);
                E.push_back({ops.emi_data + emi_off[(size_t)p] + (size_t)(a0 - e.row0) * l, l, (int)e.col0, (int)e.ncols});
            }
            RowJob* J = jobs.data() + (size_t)t * kRowsMaxJobs;
            int k = 0;
            std::vector<bool> e_used(E.size(), false);
            for (const Opnd& lo : L) {
                int pair = -1;
                for (size_t q = 0; q < E.size() && pair < 0; ++q)
                    if (!e_used[q] && E[q].col0 == lo.col0 && E[q].nc == lo.nc) pair = (int)q;
                if (pair >= 0) e_used[(size_t)pair] = true;
                for (int c0 = 0; c0 < lo.nc; c0 += kRowsChunk)
                    J[k++] = {lo.T, pair >= 0 ? E[(size_t)pair].T : nullptr, lo.ld, pair >= 0 ? E[(size_t)pair].ld : 0,
                              lo.col0, lo.nc, c0, 0};
            }
            for (size_t q = 0; q < E.size(); ++q) {
                if (e_used[q]) continue;
                for (int c0 = 0; c0 < E[q].nc; c0 += kRowsChunk)
                    J[k++] = {nullptr, E[q].T, 0, E[q].ld, E[q].col0, E[q].nc, c0, 0};
            }
            njobs[(size_t)t] = k;
        }
        RowJob* d_jobs;
        int* d_nj;
        DTB_TRY(copy_host_ints(c, &d_jobs, jobs));
        DTB_TRY(copy_host_ints(c, &d_nj, njobs));
        ops.jobs = d_jobs;
        ops.njobs = d_nj;
    }
    ops.thr = (double)1e-10f;
    ops.has_bin = c->has_bin;
    ops.has_emi = c->has_emi;
    ops.dt_scale = m->dt_scale;
    ops.stop_step = m->stop_step;
    ops.min_ratio = m->min_ratio;
    ops.nonfinite = m->nonfinite;
    for (auto& G : m->groups) c->gain_bytes += G.bytes;
    DTB_CUDA(cudaDeviceSynchronize());
    return DTB_OK;
}

void destroy_mixed(dtb_ctx* c) {
    MixedState* m = c->mixed;
    if (!m) return;
    for (auto& gp : m->graphs)
        for (cudaGraphExec_t x : gp)
            if (x) cudaGraphExecDestroy(x);
    for (auto& io : m->io_graph) {
        if (io.x) cudaGraphExecDestroy(io.x);
        if (io.g) cudaGraphDestroy(io.g);
    }
    for (cudaEvent_t e : m->ev) cudaEventDestroy(e);
    if (m->pin_col) cudaFreeHost(m->pin_col);
    if (m->adm_pin) cudaFreeHost(m->adm_pin);
    for (cudaEvent_t e : m->adm_ev)
        if (e) cudaEventDestroy(e);
    delete m;
    c->mixed = nullptr;
}

namespace {

int mixed_flush_profile(MixedState* m) {
    if (m->prof_pending == 0) return DTB_OK;
    DTB_CUDA(cudaEventSynchronize(m->ev[(size_t)(2 * (m->prof_pending - 1) + 1)]));
    for (int k = 0; k < m->prof_pending; ++k) {
        float ms = 0;
        DTB_CUDA(cudaEventElapsedTime(&ms, m->ev[(size_t)(2 * k)], m->ev[(size_t)(2 * k + 1)]));
        m->prof_ms += ms;
    }
    m->prof_pending = 0;
    return DTB_OK;
}

// One batched step; kpos is its place in a launch sequence whose last step advances the device
// step counter by the sequence length (advance), so no kernel needs a grid-wide ticket.
int mixed_step(dtb_ctx* c, bool profile, int kpos, int advance) {
    MixedState* m = c->mixed;
    const float* Fin = m->F[m->cur];
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (profile) {
        const size_t k = (size_t)m->prof_pending * 2;
        while (m->ev.size() < k + 2) {
            cudaEvent_t e;
            DTB_CUDA(cudaEventCreate(&e));
            m->ev.push_back(e);
        }
        e0 = m->ev[k];
        e1 = m->ev[k + 1];
        DTB_CUDA(cudaEventRecord(e0, c->stream));
    }
    for (auto& G : m->groups) DTB_CUDA(launch_group_gemm(c, G, Fin));
    if (profile) {
        DTB_CUDA(cudaEventRecord(e1, c->stream));
        m->prof_n++;
        if (++m->prof_pending == 256) DTB_TRY(mixed_flush_profile(m));
    }
    DTB_CUDA(launch_mixed_rows(m->ops, Fin, m->C[m->cur], m->F[m->cur ^ 1], m->C[m->cur ^ 1], m->gstep, kpos,
                               c->stream));
    if (advance > 0) DTB_CUDA(launch_advance_step(m->gstep, advance, c->stream));
    m->cur ^= 1;
    m->host_step++;
    return DTB_OK;
}

// n consecutive batched steps from the current state buffer as one graph (captured once per
// buffer and length); the last step advances the device step counter by n.
int ensure_mixed_graph(dtb_ctx* c, int n) {
    MixedState* m = c->mixed;
    const int cur = m->cur;
    if (m->graphs[cur][(size_t)n]) return DTB_OK;
    const long long hs = m->host_step;
    cudaGraph_t gr;
    DTB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = DTB_OK;
    for (int k = 0; k < n && rc == DTB_OK; ++k) rc = mixed_step(c, false, k, k == n - 1 ? n : 0);
    cudaError_t e = cudaStreamEndCapture(c->stream, &gr);
    m->host_step = hs;
    m->cur = cur;
    if (rc != DTB_OK) return rc;
    DTB_CUDA(e);
    e = cudaGraphInstantiate(&m->graphs[cur][(size_t)n], gr, 0);
    cudaGraphDestroy(gr);
    DTB_CUDA(e);
    return DTB_OK;
}

// nsteps batched steps as graph replays: whole graphs of graph_steps steps, then one graph of
// the remainder, from whichever state buffer is current.
int run_mixed_graphs(dtb_ctx* c, int64_t nsteps) {
    MixedState* m = c->mixed;
    for (int64_t done = 0; done < nsteps;) {
        const int n = (int)std::min<int64_t>(m->graph_steps, nsteps - done);
        DTB_TRY(ensure_mixed_graph(c, n));
        DTB_CUDA(cudaGraphLaunch(m->graphs[m->cur][(size_t)n], c->stream));
        m->cur ^= n & 1;
        m->host_step += n;
        done += n;
    }
    return DTB_OK;
}

// Device error flag of earlier batched launches: read behind a call's own synchronisation.
int mixed_err_enqueue(dtb_ctx* c) {
    DTB_CUDA(cudaMemcpyAsync(c->pin_err, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    return DTB_OK;
}
int mixed_err_take(dtb_ctx* c) {  // after the stream was synchronised
    if (*c->pin_err) {
        const int e = *c->pin_err;
        *c->pin_err = 0;
        cudaMemsetAsync(c->err, 0, sizeof(int), c->stream);
        cudaStreamSynchronize(c->stream);
        set_error("a bounded device wait gave up in the batched step (kernel error flags " + std::to_string(e) + ")");
        return DTB_ETIMEOUT;
    }
    return DTB_OK;
}

// Columns the gain GEMM computes: up to the highest slot that still steps (slots are admitted
// into the lowest free slots, so this tracks the number of running solves).
int refresh_active_hi(dtb_ctx* c) {
    MixedState* m = c->mixed;
    int hi = 0;
    for (int sl = m->Buser - 1; sl >= 0; --sl)
        if (m->h_stop[(size_t)sl] > m->host_step) {
            hi = sl + 1;
            break;
        }
    if (hi != m->last_active_hi) {
        const int v = hi;  // pageable source: staged before the call returns
        DTB_CUDA(cudaMemcpyAsync(m->active_hi, &v, sizeof(int), cudaMemcpyHostToDevice, c->stream));
        m->last_active_hi = hi;
    }
    return DTB_OK;
}

int mixed_check_err(dtb_ctx* c) {
    DTB_CUDA(cudaMemcpyAsync(c->pin_err, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    if (*c->pin_err) {
        const int e = *c->pin_err;
        cudaMemsetAsync(c->err, 0, sizeof(int), c->stream);
        cudaStreamSynchronize(c->stream);
        set_error("a bounded device wait gave up in the batched step (kernel error flags " + std::to_string(e) + ")");
        return DTB_ETIMEOUT;
    }
    return DTB_OK;
}

int mixed_ready(dtb_ctx* c) {
    DTB_CHECK(c, DTB_EINVAL, "null context");
    DTB_CHECK(c->prec == DTB_MIXED, DTB_ESTATE, "not a batched (DTB_MIXED) context");
    DTB_TRY(dtb_commit(c));
    return DTB_OK;
}

}  // namespace

// Launch / finish halves of dtb_batch_run for the serving loop (contexts of different grids
// run their chunks concurrently on their own streams).
int batch_launch(dtb_ctx* c, int64_t nsteps) {
    DTB_RANGE("dtb serve chunk");
    MixedState* m = c->mixed;
    DeviceGuard g(c->device);
    c->steps_run += nsteps;
    DTB_TRY(refresh_active_hi(c));
    (void)m;
    return run_mixed_graphs(c, nsteps);
}

int batch_finish(dtb_ctx* c) {
    DeviceGuard g(c->device);
    return mixed_check_err(c);
}

// Captures, instantiates and uploads every graph dtb_batch_run replays (1 to graph_steps steps
// from either state buffer); capture enqueues nothing, so the state and the step counter are
// unchanged.
int batch_prepare(dtb_ctx* c) {
    DTB_RANGE("dtb_prepare (batched graphs)");
    MixedState* m = c->mixed;
    const int cur = m->cur;
    int rc = DTB_OK;
    for (int p = 0; p < 2 && rc == DTB_OK; ++p) {
        m->cur = p;
        for (int n = 1; n <= m->graph_steps && rc == DTB_OK; ++n) rc = ensure_mixed_graph(c, n);
    }
    m->cur = cur;
    if (rc != DTB_OK) return rc;
    for (auto& gp : m->graphs)
        for (cudaGraphExec_t x : gp)
            if (x) DTB_CUDA(cudaGraphUpload(x, c->stream));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    return DTB_OK;
}

int batch_capacity(dtb_ctx* c) { return c->mixed ? c->mixed->Buser : 0; }

namespace dtb {
std::string batch_profile_json(const dtb_ctx* c) {
    const MixedState* m = c->mixed;
    if (!m) return "\"batch\": 0";
    std::string js = "\"batch\": " + std::to_string(m->Buser) + ", \"batched_steps\": " + std::to_string(m->host_step);
    if (m->prof_n > 0) {
        char b[64];
        std::snprintf(b, sizeof(b), "%.6g", m->prof_ms / (double)m->prof_n);
        js += std::string(", \"gemm_avg_ms_per_step\": ") + b;
    }
    js += ", \"gemm_plans\": [";
    for (size_t i = 0; i < m->groups.size(); ++i) {
        const MixedGroup& G = m->groups[i];
        char b[160];
        std::snprintf(b, sizeof(b), "%s{\"M\": %d, \"pair\": %d, \"bn\": %d, \"n_splits\": %d, \"tuned_us\": %.4g}",
                      i ? ", " : "", G.M, G.pair ? 1 : 0, G.bn, G.n_splits, G.tuned_us);
        js += b;
    }
    return js + "]";
}
}  // namespace dtb
long long batch_step(dtb_ctx* c) { return c->mixed ? c->mixed->host_step : 0; }

extern "C" {

int32_t dtb_batch_admit(dtb_ctx* c, int32_t slot, const double* f0, double dt_scale, int64_t n_steps) {
    DTB_RANGE("dtb_batch_admit");
    DTB_TRY(mixed_ready(c));
    MixedState* m = c->mixed;
    DTB_CHECK(slot >= 0 && slot < m->Buser, DTB_ENOTFOUND, "dtb_batch_admit: slot out of range");
    DTB_CHECK(f0, DTB_EINVAL, "dtb_batch_admit: null f0");
    DTB_CHECK(n_steps >= 0 && std::isfinite(dt_scale), DTB_EINVAL, "dtb_batch_admit: bad dt_scale or step count");
    DeviceGuard g(c->device);
    const int n = (int)c->n_state, B = m->Bcap;
    // the next staging record of the ring, free once its previous scatter has run
    const AdmitRecord R = admit_record(n, c->ns);
    const int k = m->adm_next;
    m->adm_next = (k + 1) % kAdmitRing;
    DTB_CUDA(cudaEventSynchronize(m->adm_ev[k]));
    unsigned char* rec = m->adm_pin + (size_t)k * R.bytes;
    float* fcol = reinterpret_cast<float*>(rec + R.f);
    float* ccol = reinterpret_cast<float*>(rec + R.c);
    for (int i = 0; i < n; ++i) {
        fcol[i] = (float)f0[i];
        ccol[i] = (float)(f0[i] - (double)(float)f0[i]);  // exact remainder as the compensation
    }
    // power-of-two species scales from the initial spectrum: X uses f * 2^-e
    float* sg = reinterpret_cast<float*>(rec + R.sig);
    float* isg = reinterpret_cast<float*>(rec + R.isig);
    for (int sp = 0; sp < c->ns; ++sp) {
        double mx = 0;
        for (int cl = 0; cl < c->n_space; ++cl)
            for (int64_t q = c->off[sp]; q < c->off[sp + 1]; ++q) mx = std::max(mx, std::fabs(f0[cl * c->n_mom + q]));
        int ex = 0;
        if (mx > 0 && std::isfinite(mx)) std::frexp(mx, &ex);
        sg[sp] = std::ldexp(1.0f, ex);
        isg[sp] = std::ldexp(1.0f, -ex);
    }
    const long long stop = m->host_step + n_steps;
    *reinterpret_cast<double*>(rec + R.dt) = dt_scale;
    *reinterpret_cast<long long*>(rec + R.stop) = stop;
    unsigned char* drec = m->adm_dev + (size_t)k * R.bytes;
    DTB_CUDA(cudaMemcpyAsync(drec, rec, R.bytes, cudaMemcpyHostToDevice, c->stream));
    DTB_CUDA(launch_admit_slot(drec, n, c->ns, slot, B, m->F[m->cur], m->C[m->cur], m->sig, m->isig, m->dt_scale,
                               m->stop_step, m->min_ratio, m->nonfinite, ord_enc_host(INFINITY), c->stream));
    DTB_CUDA(cudaEventRecord(m->adm_ev[k], c->stream));
    m->h_stop[(size_t)slot] = stop;
    m->h_start[(size_t)slot] = m->host_step;
    return DTB_OK;
}

int32_t dtb_batch_run(dtb_ctx* c, int64_t nsteps) {
    DTB_RANGE("dtb_batch_run");
    DTB_TRY(mixed_ready(c));
    DTB_CHECK(nsteps >= 0, DTB_EINVAL, "dtb_batch_run: nsteps < 0");
    MixedState* m = c->mixed;
    DeviceGuard g(c->device);
    c->steps_run += nsteps;
    DTB_TRY(refresh_active_hi(c));
    if (m->profiling) {
        for (int64_t done = 0; done < nsteps; ++done) DTB_TRY(mixed_step(c, true, 0, 1));
        DTB_TRY(mixed_flush_profile(m));
        return mixed_check_err(c);
    }
    // enqueued only: a device error surfaces at the next call that reads results
    return run_mixed_graphs(c, nsteps);
}

namespace {

// Every slot's f from the caller's host array into the state pair (F, C), enqueued.
int upload_all(dtb_ctx* c, const double* f) {
    MixedState* m = c->mixed;
    const int n = (int)c->n_state;
    const size_t bytes = sizeof(double) * (size_t)n * m->Buser;
    if (!m->io_all) DTB_TRY(c->alloc(&m->io_all, bytes));
    DTB_CUDA(cudaMemcpyAsync(m->io_all, f, bytes, cudaMemcpyHostToDevice, c->stream));
    DTB_CUDA(launch_pack_f(m->io_all, m->Buser, n, m->Bcap, m->F[m->cur], m->C[m->cur], c->stream));
    return DTB_OK;
}

// Every slot's f (F + C in FP64) into the caller's host array, enqueued.
int download_all(dtb_ctx* c, double* f) {
    MixedState* m = c->mixed;
    const int n = (int)c->n_state;
    const size_t bytes = sizeof(double) * (size_t)n * m->Buser;
    if (!m->io_all) DTB_TRY(c->alloc(&m->io_all, bytes));
    DTB_CUDA(launch_unpack_f(m->F[m->cur], m->C[m->cur], m->Buser, n, m->Bcap, m->io_all, c->stream));
    DTB_CUDA(cudaMemcpyAsync(f, m->io_all, bytes, cudaMemcpyDeviceToHost, c->stream));
    return DTB_OK;
}

}  // namespace

namespace {

bool page_locked(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// One step's host round trip (f in, one batched step, f out, the error flag) as a graph for the
// current state buffer, captured once and then replayed with the caller's host addresses
// patched into its two copy nodes.
int run_io_graph(dtb_ctx* c, const double* f_in, double* f_out) {
    MixedState* m = c->mixed;
    const int n = (int)c->n_state;
    const size_t bytes = sizeof(double) * (size_t)n * m->Buser;
    if (!m->io_all) DTB_TRY(c->alloc(&m->io_all, bytes));
    DTB_TRY(refresh_active_hi(c));
    MixedState::IoGraph& io = m->io_graph[m->cur];
    if (!io.x) {
        const int cur = m->cur;
        const long long hs = m->host_step;
        cudaGraph_t gr = nullptr;
        DTB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = upload_all(c, f_in);
        if (rc == DTB_OK) rc = mixed_step(c, false, 0, 1);
        if (rc == DTB_OK) rc = download_all(c, f_out);
        if (rc == DTB_OK) rc = mixed_err_enqueue(c);
        cudaError_t e = cudaStreamEndCapture(c->stream, &gr);
        m->cur = cur;
        m->host_step = hs;
        if (rc != DTB_OK) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
        }
        DTB_CUDA(e);
        size_t nn = 0;
        DTB_CUDA(cudaGraphGetNodes(gr, nullptr, &nn));
        std::vector<cudaGraphNode_t> nodes(nn);
        DTB_CUDA(cudaGraphGetNodes(gr, nodes.data(), &nn));
        for (cudaGraphNode_t nd : nodes) {
            cudaGraphNodeType t;
            DTB_CUDA(cudaGraphNodeGetType(nd, &t));
            if (t != cudaGraphNodeTypeMemcpy) continue;
            cudaMemcpy3DParms p{};
            DTB_CUDA(cudaGraphMemcpyNodeGetParams(nd, &p));
            // the upload lands in the device staging array, the download leaves it
            if (p.dstPtr.ptr == m->io_all) io.h2d = nd;
            if (p.srcPtr.ptr == m->io_all) io.d2h = nd;
        }
        if (!io.h2d || !io.d2h) {
            cudaGraphDestroy(gr);
            set_error("dtb_batch_run_io: the round-trip graph has no state copies");
            return DTB_ECUDA;
        }
        e = cudaGraphInstantiate(&io.x, gr, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(gr);
            io.x = nullptr;
            DTB_CUDA(e);
        }
        io.g = gr;
        io.src = f_in;
        io.dst = f_out;
    }
    if (io.src != f_in) {
        DTB_CUDA(cudaGraphExecMemcpyNodeSetParams1D(io.x, io.h2d, m->io_all, f_in, bytes, cudaMemcpyHostToDevice));
        io.src = f_in;
    }
    if (io.dst != f_out) {
        DTB_CUDA(cudaGraphExecMemcpyNodeSetParams1D(io.x, io.d2h, f_out, m->io_all, bytes, cudaMemcpyDeviceToHost));
        io.dst = f_out;
    }
    DTB_CUDA(cudaGraphLaunch(io.x, c->stream));
    m->cur ^= 1;
    m->host_step++;
    c->steps_run++;
    return DTB_OK;
}

}  // namespace

int32_t dtb_batch_run_io(dtb_ctx* c, const double* f_in, int64_t nsteps, double* f_out) {
    DTB_RANGE("dtb_batch_run_io");
    DTB_TRY(mixed_ready(c));
    DTB_CHECK(nsteps >= 0, DTB_EINVAL, "dtb_batch_run_io: nsteps < 0");
    DeviceGuard g(c->device);
    MixedState* m = c->mixed;
    if (nsteps == 1 && f_in && f_out && !m->profiling && page_locked(f_in) && page_locked(f_out)) {
        DTB_TRY(run_io_graph(c, f_in, f_out));
        DTB_CUDA(cudaStreamSynchronize(c->stream));  // one wait for the whole round trip
        DTB_TRY(mixed_err_take(c));
        return DTB_OK;
    }
    if (f_in) DTB_TRY(upload_all(c, f_in));
    if (nsteps > 0) DTB_TRY(dtb_batch_run(c, nsteps));
    if (f_out) DTB_TRY(download_all(c, f_out));
    DTB_TRY(mixed_err_enqueue(c));
    DTB_CUDA(cudaStreamSynchronize(c->stream));  // one wait for the whole round trip
    DTB_TRY(mixed_err_take(c));
    return DTB_OK;
}

int32_t dtb_batch_get_f(dtb_ctx* c, int32_t slot, double* f) {
    DTB_TRY(mixed_ready(c));
    MixedState* m = c->mixed;
    DTB_CHECK(slot >= 0 && slot < m->Buser, DTB_ENOTFOUND, "dtb_batch_get_f: slot out of range");
    DTB_CHECK(f, DTB_EINVAL, "dtb_batch_get_f: null output");
    DeviceGuard g(c->device);
    const int n = (int)c->n_state, B = m->Bcap;
    DTB_CUDA(cudaMemcpy2DAsync(m->pin_col, sizeof(float), m->F[m->cur] + slot, sizeof(float) * B, sizeof(float), n,
                               cudaMemcpyDeviceToHost, c->stream));
    DTB_CUDA(cudaMemcpy2DAsync(m->pin_col + n, sizeof(float), m->C[m->cur] + slot, sizeof(float) * B, sizeof(float), n,
                               cudaMemcpyDeviceToHost, c->stream));
    DTB_TRY(mixed_err_enqueue(c));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    DTB_TRY(mixed_err_take(c));
    for (int i = 0; i < n; ++i) f[i] = (double)m->pin_col[i] + (double)m->pin_col[n + i];
    return DTB_OK;
}

int32_t dtb_batch_slot_info(dtb_ctx* c, int32_t slot, int64_t* steps_done, int64_t* steps_left, double* cr_max,
                            int32_t* finite) {
    DTB_TRY(mixed_ready(c));
    MixedState* m = c->mixed;
    DTB_CHECK(slot >= 0 && slot < m->Buser, DTB_ENOTFOUND, "dtb_batch_slot_info: slot out of range");
    DeviceGuard g(c->device);
    const long long stop = m->h_stop[(size_t)slot];
    const long long now = std::min(m->host_step, stop);
    if (steps_done) *steps_done = std::max(0LL, now - m->h_start[(size_t)slot]);
    if (steps_left) *steps_left = std::max(0LL, stop - m->host_step);
    if (cr_max || finite) {
        unsigned long long e = 0;
        int nf = 0;
        DTB_CUDA(cudaMemcpyAsync(&e, m->min_ratio + slot, sizeof(e), cudaMemcpyDeviceToHost, c->stream));
        DTB_CUDA(cudaMemcpyAsync(&nf, m->nonfinite + slot, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        DTB_TRY(mixed_err_enqueue(c));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
        DTB_TRY(mixed_err_take(c));
        if (cr_max) *cr_max = -ord_dec_host(e);
        if (finite) *finite = nf ? 0 : 1;
    }
    return DTB_OK;
}

int32_t dtb_batch_release(dtb_ctx* c, int32_t slot) {
    DTB_TRY(mixed_ready(c));
    MixedState* m = c->mixed;
    DTB_CHECK(slot >= 0 && slot < m->Buser, DTB_ENOTFOUND, "dtb_batch_release: slot out of range");
    DeviceGuard g(c->device);
    const long long zero = 0;
    DTB_CUDA(cudaMemcpyAsync(m->stop_step + slot, &zero, sizeof(zero), cudaMemcpyHostToDevice, c->stream));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    m->h_stop[(size_t)slot] = 0;
    return DTB_OK;
}

int32_t dtb_batch_set_f_all(dtb_ctx* c, const double* f) {
    DTB_TRY(mixed_ready(c));
    DTB_CHECK(f, DTB_EINVAL, "dtb_batch_set_f_all: null input");
    DeviceGuard g(c->device);
    DTB_TRY(upload_all(c, f));
    DTB_CUDA(cudaStreamSynchronize(c->stream));  // the caller may reuse f on return
    return DTB_OK;
}

int32_t dtb_batch_get_f_all(dtb_ctx* c, double* f) {
    DTB_TRY(mixed_ready(c));
    DTB_CHECK(f, DTB_EINVAL, "dtb_batch_get_f_all: null output");
    DeviceGuard g(c->device);
    DTB_TRY(download_all(c, f));
    DTB_TRY(mixed_err_enqueue(c));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    DTB_TRY(mixed_err_take(c));
    return DTB_OK;
}

int32_t dtb_batch_moments(dtb_ctx* c, const double* w, double* number, double* energy) {
    DTB_TRY(mixed_ready(c));
    DTB_CHECK(w && number && energy, DTB_EINVAL, "dtb_batch_moments: null argument");
    MixedState* m = c->mixed;
    DeviceGuard g(c->device);
    const int B = m->Bcap, ns = c->ns;
    DTB_CUDA(cudaMemcpyAsync(m->mom_w, w, sizeof(double) * (size_t)c->n_mom, cudaMemcpyHostToDevice, c->stream));
    DTB_CUDA(launch_batch_moments(m->F[m->cur], m->C[m->cur], B, m->sp_off, ns, (int)c->n_mom, c->n_space, m->mom_w,
                                  m->mom_out, c->stream));
    std::vector<double> out((size_t)2 * ns * B * c->n_space);
    DTB_CUDA(cudaMemcpyAsync(out.data(), m->mom_out, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, c->stream));
    DTB_TRY(mixed_err_enqueue(c));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    DTB_TRY(mixed_err_take(c));
    for (size_t k = 0; k < (size_t)m->Buser * c->n_space * ns; ++k) {
        number[k] = out[2 * k];
        energy[k] = out[2 * k + 1];
    }
    return DTB_OK;
}

int32_t dtb_batch_capacity(dtb_ctx* c, int32_t* capacity, int64_t* step) {
    DTB_TRY(mixed_ready(c));
    if (capacity) *capacity = c->mixed->Buser;
    if (step) *step = c->mixed->host_step;
    return DTB_OK;
}

int32_t dtb_batch_set_profiling(dtb_ctx* c, int32_t on) {
    DTB_TRY(mixed_ready(c));
    MixedState* m = c->mixed;
    if (m->profiling && m->prof_pending) DTB_TRY(mixed_flush_profile(m));
    m->profiling = on != 0;
    m->prof_ms = 0;
    m->prof_n = 0;
    m->prof_pending = 0;
    return DTB_OK;
}

int32_t dtb_set_tune_cache(const char* path) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plans.clear();
    g_plan_file = path ? path : "";
    if (!path) return DTB_OK;
    if (FILE* f = std::fopen(path, "r")) {
        char key[160];
        GemmPlan p;
        while (std::fscanf(f, "%159s %d %d %d %lf", key, &p.pair, &p.bn, &p.splits, &p.us) == 5) g_plans[key] = p;
        std::fclose(f);
    }
    return DTB_OK;
}

int32_t dtb_batch_gemm_plan(dtb_ctx* c, int32_t group, int32_t* pair, int32_t* bn, int32_t* n_splits,
                            double* tuned_us) {
    DTB_TRY(mixed_ready(c));
    MixedState* m = c->mixed;
    DTB_CHECK(group >= 0, DTB_EINVAL, "negative group index");
    if (group >= (int32_t)m->groups.size()) return DTB_ENOTFOUND;
    const MixedGroup& G = m->groups[(size_t)group];
    if (pair) *pair = G.pair ? 1 : 0;
    if (bn) *bn = G.bn;
    if (n_splits) *n_splits = G.n_splits;
    if (tuned_us) *tuned_us = G.tuned_us;
    return DTB_OK;
}

int32_t dtb_batch_gemm_stats(dtb_ctx* c, double* avg_ms, double* flops_per_step, double* bytes_per_step,
                             int32_t* launches_per_step) {
    DTB_TRY(mixed_ready(c));
    MixedState* m = c->mixed;
    double fl = 0, by = 0;
    for (auto& G : m->groups) {
        fl += G.flops;
        by += G.bytes;
    }
    if (avg_ms) *avg_ms = m->prof_n ? m->prof_ms / (double)m->prof_n : 0.0;
    if (flops_per_step) *flops_per_step = fl;
    if (bytes_per_step) *bytes_per_step = by;
    if (launches_per_step) *launches_per_step = (int32_t)m->groups.size() + 1;  // + advance_step per graph
    return DTB_OK;
}

}  // extern "C"
