// The context behind dtb_ctx* and the helpers shared by the runtime translation units.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "dtb_internal.h"

using namespace dtb;

#define DTB_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_) + " (" __FILE__ ":" + \
                      std::to_string(__LINE__) + ")");                                        \
            return e_ == cudaErrorMemoryAllocation ? DTB_ENOMEM : DTB_ECUDA;                  \
        }                                                                                     \
    } while (0)

#define DTB_CHECK(cond, code, msg) \
    do {                           \
        if (!(cond)) {             \
            set_error(msg);        \
            return (code);         \
        }                          \
    } while (0)

namespace dtb {

constexpr int kProfRing = 256;
constexpr int64_t kMaxScheduleSteps = 100000000;
constexpr int kMaxGraphSteps = 1024;  // steps per captured graph (dtb_opts.graph_steps)

// An NVTX range over a host entry point (upload, commit, steps, graph replays, serving chunks):
// visible on a profiler timeline, a no-op without one.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
#define DTB_RANGE_CAT2(a, b) a##b
#define DTB_RANGE_CAT(a, b) DTB_RANGE_CAT2(a, b)
#define DTB_RANGE(name) ::dtb::NvtxRange DTB_RANGE_CAT(dtb_range_, __LINE__)(name)

// Path of the run summary each context appends at dtb_destroy (environment DTB_PROFILE), or null.
const char* profile_path();
// The batched context's part of that summary (batch_api.cpp): JSON members without braces.
std::string batch_profile_json(const dtb_ctx* c);

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

struct GainStage {
    int out, in1, in2;
    std::vector<double> host;  // [no][n1][n2], FP64 sum of all host uploads
    std::vector<std::pair<const void*, int>> dev_src;  // device sources (pointer, dtype), added in order
};

// Gain block entries from a sparse M_Bin: COO with local (output row, b, c) indices.
struct SparseGain {
    std::vector<int32_t> a, b, c;
    std::vector<double> v;
};

struct EmiPiece {
    int64_t row0, nrows, col0, ncols;
    std::vector<double> data;  // row-major
};

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

struct MixedState;

}  // namespace dtb

struct dtb_ctx {
    long long steps_run = 0;  // steps launched over the context's life (the DTB_PROFILE summary)
    dtb_dims dims{};
    dtb_opts opts{};
    int ns = 0;
    int64_t sz[DTB_MAX_SPECIES]{};
    int64_t off[DTB_MAX_SPECIES + 1]{};
    int64_t offp[DTB_MAX_SPECIES + 1]{};
    int64_t n_mom = 0, n_state = 0;
    int n_space = 1;
    int prec = DTB_F64;
    size_t esz = 8;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // host staging
    std::map<std::tuple<int, int, int>, GainStage> gains;
    std::map<std::tuple<int, int, int>, SparseGain> sgains;  // from dtb_upload_mbin_csc
    std::vector<std::vector<char>> sparse_stage;              // commit-time host data of sparse blocks
    std::map<std::pair<int, int>, std::vector<double>> losses;
    std::vector<EmiPiece> emis;
    std::vector<int64_t> flux_r, flux_c;
    std::vector<double> flux_v;
    bool symplectic = false;             // ForwardSymplecticEuler: X kept apart from P
    std::vector<int64_t> xflux_r, xflux_c;
    std::vector<double> xflux_v;
    void* fm_buf = nullptr;              // f_Momentum of the symplectic step
    void* dfm_buf = nullptr;             // df_Momentum of the symplectic step
    std::vector<double> Ap, Vol, f_init, inj;
    bool have_vectors = false;
    bool has_bin_domain = false;         // BinM.Domain !== nothing
    std::vector<int64_t> bin_domain;     // its off_space entries
    int n_bin_cells = 0;                 // cells the gain kernel runs (domain cells, or all)
    int* bin_cells = nullptr;            // device list of those cells (null: 0..n_space-1)
    bool committed = false;

    // device memory
    std::vector<void*> allocs;
    size_t dev_bytes = 0;
    void* G_all = nullptr;
    double gain_bytes = 0;  // algorithmic gain bytes per step (one read of every G element)
    GainUnit* units = nullptr;
    int n_units = 0;
    int gain_grid = 0;
    int f_smem_len = 0;
    int* unit_ptr = nullptr;
    double* partial = nullptr;
    void* f_buf[2] = {nullptr, nullptr};
    void* f_init_dev = nullptr;
    int cur = 0;
    double* dt_arr = nullptr;
    long long hist_cap = 65536;
    unsigned long long* ctr = nullptr;
    unsigned long long host_ctr = 0;
    StepDiagDev* hist = nullptr;
    // row-block diagnostics records: [graph_steps][rows_grid][kStepRecFields], slot k for step k
    // of a sequence
    double* blk_red = nullptr;
    int rows_grid = 0;
    unsigned* ticket = nullptr;
    long long launches = 0;      // kernels the step functions have launched (graph replays count their nodes)
    long long graph_launches = 0;  // kernel nodes of the step graph
    int* err = nullptr;
    int* sp_off_dev = nullptr;
    double* mom_w = nullptr;
    double* mom_out = nullptr;
    int sp_off_host[2 * DTB_MAX_SPECIES + 2]{};
    RowOps<double> ops_d{};
    RowOps<float> ops_f{};
    bool has_bin = false, has_emi = false;
    MixedState* mixed = nullptr;  // batched mixed-precision state (precision DTB_MIXED)

    // pinned staging
    double* pin_dt = nullptr;
    StepDiagDev* pin_hist = nullptr;
    int* pin_err = nullptr;
    float* pin_f32 = nullptr;  // FP32 state staging for dtb_get_f / dtb_set_f

    // pipelined Solve (allocated on first use): dt staging and diagnostics read-back, double
    // buffered; a ring of save slots on the device and in pinned memory; a copy stream
    double* pin_dt2 = nullptr;          // [2][hist_cap]
    StepDiagDev* pin_hist2 = nullptr;   // [2][hist_cap]
    void* save_dev = nullptr;           // [kSaveRing][n_state] state elements
    void* save_pin = nullptr;           // [kSaveRing][n_state]
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t pipe_ev[16] = {};       // dt staging x2, hist x2, saved x kSaveRing, landed x kSaveRing
    bool pipe_ready = false;

    // graphs
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 16;  // set at creation (the plain path's default depends on the grid size)
    int graph_verbose = -1;

    // profiling
    bool profiling = false;
    double prof_ms = 0.0;
    long long prof_n = 0;
    int prof_pending = 0;
    std::vector<cudaEvent_t> ev;

    template <typename P>
    int alloc(P** p, size_t bytes) {
        void* q = nullptr;
        if (bytes == 0) bytes = 16;
        cudaError_t e = cudaMalloc(&q, bytes);
        if (e != cudaSuccess) {
            set_error("cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
            return DTB_ENOMEM;
        }
        allocs.push_back(q);
        dev_bytes += bytes;
        *p = reinterpret_cast<P*>(q);
        return DTB_OK;
    }
    void free_all() {
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        dev_bytes = 0;
    }
};

#define DTB_TRY(expr)              \
    do {                           \
        int rc_ = (expr);          \
        if (rc_ != DTB_OK) return rc_; \
    } while (0)


template <typename T>
inline int copy_host_vec(dtb_ctx* c, T** dst, const std::vector<double>& src) {
    std::vector<T> tmp(src.size());
    for (size_t i = 0; i < src.size(); ++i) tmp[i] = (T)src[i];
    DTB_TRY(c->alloc(dst, sizeof(T) * std::max<size_t>(1, tmp.size())));
    if (!tmp.empty()) {
        DTB_CUDA(cudaMemcpyAsync(*dst, tmp.data(), sizeof(T) * tmp.size(), cudaMemcpyHostToDevice, c->stream));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
    }
    return DTB_OK;
}

template <typename I>
inline int copy_host_ints(dtb_ctx* c, I** dst, const std::vector<I>& src) {
    DTB_TRY(c->alloc(dst, sizeof(I) * std::max<size_t>(1, src.size())));
    if (!src.empty()) {
        DTB_CUDA(cudaMemcpyAsync(*dst, src.data(), sizeof(I) * src.size(), cudaMemcpyHostToDevice, c->stream));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
    }
    return DTB_OK;
}


inline int species_of(const dtb_ctx* c, int64_t a) {
    int s = 0;
    while (s + 1 < c->ns && a >= c->off[s + 1]) ++s;
    return s;
}
