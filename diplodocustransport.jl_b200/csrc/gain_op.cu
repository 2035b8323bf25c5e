// Kernel-level entry for one gain block held in the caller's device memory:
//   out[a] = sum_b f1[b] sum_c G[a][b][c] f2[c]
// i.e. the two products of update_Big_Bin! (SteppingMethods.jl:372-373) restricted to one
// (output species, input-1 species, input-2 species) block, without the context API.
// It runs the same gain_stream kernel as the stepping path, followed by a per-row sum of the
// per-unit partials.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <mutex>
#include <string>

#include "dtb_internal.h"

namespace dtb {

__global__ void row_sums_kernel(const double* __restrict__ partial, int n_rows, int splits, double* __restrict__ out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_rows) return;
    double s = 0.0;
    for (int j = 0; j < splits; ++j) s += partial[(size_t)a * splits + j];
    out[a] = s;
}

cudaError_t launch_row_sums(const double* partial, int n_rows, int splits, double* out, cudaStream_t s) {
    row_sums_kernel<<<(n_rows + 255) / 256, 256, 0, s>>>(partial, n_rows, splits, out);
    return cudaGetLastError();
}

// The work table of one contraction, written on the device: unit u = a * splits + j covers
// output row a over b-rows [j * nb, min(n1, (j + 1) * nb)). Nothing in the stream reads host
// memory, so the inputs of a call are only the caller's device arrays.
__global__ void gain_op_units_kernel(GainUnit* __restrict__ units, long long n_units, int splits, long long n1,
                                     long long n2, long long nb, int tile_b, int c_off) {
    const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_units) return;
    const long long a = u / splits;
    const long long b0 = (u - a * splits) * nb;
    GainUnit g;
    g.g_off = (a * n1 + b0) * n2;
    g.b_off = (int)b0;
    g.c_off = c_off;
    g.nb = (int)(nb < n1 - b0 ? nb : n1 - b0);
    g.n2p = (int)n2;
    g.tile_b = tile_b;
    g.row = (int)a;
    units[u] = g;
}

int gain_op_plan(int64_t n_out, int64_t n1, int64_t n2, int esz, int num_sms, int bps, GainOpPlan& plan) {
    const int64_t row_b = n2 * esz;
    if (n2 <= 0 || n2 % 8 != 0 || row_b > kGainTileBytes) {
        set_error("gain op: n2 must be a positive multiple of 8 with n2 * element size <= 16384 bytes");
        return DTB_EINVAL;
    }
    if (n_out <= 0 || n1 <= 0 || n_out > INT32_MAX || n1 > INT32_MAX / 2) {
        set_error("gain op: n_out and n1 must be positive (and below 2^31, 2^30)");
        return DTB_EINVAL;
    }
    const double tot = (double)n_out * n1 * n2 * esz;
    const double target =
        std::min(256.0 * 1024, std::max((double)kGainTileBytes, tot / ((double)num_sms * std::max(1, bps) * 8)));
    plan.tile_b = (int)std::max<int64_t>(1, std::min<int64_t>(n1, kGainTileBytes / row_b));
    plan.nb = std::max<int64_t>(plan.tile_b, (int64_t)(target / row_b) / plan.tile_b * plan.tile_b);
    plan.splits = (int)((n1 + plan.nb - 1) / plan.nb);
    plan.n_units = n_out * plan.splits;
    if (plan.n_units > INT32_MAX) {
        set_error("gain op: more than 2^31 work units");
        return DTB_EINVAL;
    }
    return DTB_OK;
}

int gain_op_check_args(const char* who, int32_t dtype, const void* G, const void* f1, const void* f2,
                       const double* out) {
    if (!G || !f1 || !f2 || !out) {
        set_error(std::string(who) + ": null argument");
        return DTB_EINVAL;
    }
    if (dtype != DTB_DTYPE_F64 && dtype != DTB_DTYPE_F32) {
        set_error(std::string(who) + ": bad dtype");
        return DTB_EINVAL;
    }
    // G is read with bulk copies (16-byte aligned source addresses), out with FP64 stores;
    // f1 and f2 are copied with cudaMemcpyAsync and only need their element alignment
    const size_t esz = dtype == DTB_DTYPE_F64 ? 8 : 4;
    if ((uintptr_t)G % 16 != 0 || (uintptr_t)out % 8 != 0 || (uintptr_t)f1 % esz != 0 || (uintptr_t)f2 % esz != 0) {
        set_error(std::string(who) + ": G must be 16-byte aligned, out 8-byte aligned and f1, f2 aligned to "
                  "their element size");
        return DTB_EINVAL;
    }
    return DTB_OK;
}

int gain_op_read_flag(const char* who, int* err, cudaStream_t s) {
    int h = 0;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && h) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e == cudaSuccess && h) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(std::string(who) + ": " + cudaGetErrorString(e));
        return DTB_ECUDA;
    }
    if (h & (KERR_TIMEOUT_FULL | KERR_TIMEOUT_EMPTY | KERR_TIMEOUT_DRAIN)) {
        set_error(std::string(who) + ": a bounded device wait gave up (kernel error flags " + std::to_string(h) +
                  "); the result of that contraction is incomplete");
        return DTB_ETIMEOUT;
    }
    if (h) {
        set_error(std::string(who) + ": a work unit failed its bounds check (kernel error flags " +
                  std::to_string(h) + ")");
        return DTB_EINVAL;
    }
    return DTB_OK;
}

// Runs the contraction with scratch at `scratch` (units, then partials, then the f1|f2 vector).
// The kernel error flag `err` is cleared first, in stream order.
int gain_op_run(int32_t dtype, const void* G, int64_t n_out, int64_t n1, int64_t n2, const void* f1, const void* f2,
                double* out, const GainOpPlan& plan, unsigned char* scratch, int* err, cudaStream_t s) {
    const int esz = dtype == DTB_DTYPE_F64 ? 8 : 4;
    const int n_units = (int)plan.n_units;
    const size_t units_bytes = ((size_t)n_units * sizeof(GainUnit) + 255) / 256 * 256;
    const size_t part_bytes = ((size_t)n_units * sizeof(double) + 255) / 256 * 256;
    GainUnit* d_units = reinterpret_cast<GainUnit*>(scratch);
    double* d_part = reinterpret_cast<double*>(scratch + units_bytes);
    unsigned char* d_f = scratch + units_bytes + part_bytes;
    const int64_t offp1 = (n1 + 7) / 8 * 8;
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e == cudaSuccess) {
        gain_op_units_kernel<<<(unsigned)((n_units + 255) / 256), 256, 0, s>>>(d_units, n_units, plan.splits, n1, n2,
                                                                            plan.nb, plan.tile_b, (int)offp1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_f, f1, (size_t)n1 * esz, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_f + n1 * esz, f2, (size_t)n2 * esz, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) {
        set_error(std::string("gain op: set-up in scratch failed: ") + cudaGetErrorString(e));
        return DTB_ECUDA;
    }
    // f1|f2 stored unpadded as a two-species state [0, n1) [n1, n1 + n2); the kernel stages it
    // padded ([0, offp1) [offp1, offp1 + n2)) in shared memory
    int sp[6] = {0, (int)n1, (int)(n1 + n2), 0, (int)offp1, (int)(offp1 + n2)};
    const int f_len = (int)(offp1 + n2);
    const int n_state = (int)(n1 + n2);
    const int bps = gain_stream_blocks_per_sm(esz, f_len);
    if (bps < 1) {
        set_error("gain op: vectors too long for the shared-memory stage");
        return DTB_EINVAL;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::max(1, std::min(n_units, sms * bps));
    if (dtype == DTB_DTYPE_F64)
        e = launch_gain_stream<double>(static_cast<const double*>(G), d_units, n_units,
                                       reinterpret_cast<const double*>(d_f), n_state, sp, 2, f_len, d_part, 1, grid, err, s);
    else
        e = launch_gain_stream<float>(static_cast<const float*>(G), d_units, n_units,
                                      reinterpret_cast<const float*>(d_f), n_state, sp, 2, f_len, d_part, 1, grid, err, s);
    if (e == cudaSuccess) e = launch_row_sums(d_part, (int)n_out, plan.splits, out, s);
    if (e != cudaSuccess) {
        set_error(std::string("gain op: launch failed: ") + cudaGetErrorString(e));
        return DTB_ECUDA;
    }
    return DTB_OK;
}

size_t gain_op_scratch_bytes(int64_t n_units, int64_t n1, int64_t n2, int esz) {
    return ((size_t)n_units * sizeof(GainUnit) + 255) / 256 * 256 + ((size_t)n_units * 8 + 255) / 256 * 256 +
           (size_t)(n1 + n2) * esz;
}

}  // namespace dtb

using namespace dtb;

namespace {
// Scratch of dtb_gain_contract: one buffer per device, grown on demand, kept until exit.
struct OpScratch {
    unsigned char* p = nullptr;
    size_t bytes = 0;
    int* err = nullptr;
};
std::mutex g_op_mu;
OpScratch g_op[64];

int* op_flag(int dev) {
    std::lock_guard<std::mutex> lk(g_op_mu);
    return g_op[dev].err;
}
}  // namespace

namespace dtb {
int* noalloc_flag(int dev);  // gain_noalloc.cu: nullptr before the entry's set-up on `dev`
}

extern "C" int32_t dtb_gain_contract(int32_t dtype, const void* G, int64_t n_out, int64_t n1, int64_t n2,
                                     const void* f1, const void* f2, double* out, void* stream) {
    int rc = gain_op_check_args("dtb_gain_contract", dtype, G, f1, f2, out);
    if (rc != DTB_OK) return rc;
    const int esz = dtype == DTB_DTYPE_F64 ? 8 : 4;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("dtb_gain_contract: no current CUDA device");
        return DTB_ENODEV;
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    GainOpPlan plan;
    rc = gain_op_plan(n_out, n1, n2, esz, sms, gain_stream_blocks_per_sm(esz, (int)((n1 + 7) / 8 * 8 + n2)), plan);
    if (rc != DTB_OK) return rc;
    const size_t need = gain_op_scratch_bytes(plan.n_units, n1, n2, esz);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(g_op_mu);
    OpScratch& sc = g_op[dev];
    if (sc.bytes < need) {
        cudaStreamSynchronize(s);
        if (sc.p) cudaFree(sc.p);
        sc.p = nullptr;
        sc.bytes = 0;
        cudaError_t e = cudaMalloc(&sc.p, need);
        if (e != cudaSuccess) {
            set_error(std::string("dtb_gain_contract: scratch allocation failed: ") + cudaGetErrorString(e));
            return DTB_ENOMEM;
        }
        sc.bytes = need;
    }
    if (!sc.err && cudaMalloc(&sc.err, sizeof(int)) != cudaSuccess) {
        sc.err = nullptr;
        set_error("dtb_gain_contract: error-flag allocation failed");
        return DTB_ENOMEM;
    }
    return gain_op_run(dtype, G, n_out, n1, n2, f1, f2, out, plan, sc.p, sc.err, s);
}

extern "C" int32_t dtb_gain_contract_status(void* stream) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("dtb_gain_contract_status: no current CUDA device");
        return DTB_ENODEV;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int rc = DTB_OK;
    if (int* f = op_flag(dev)) rc = gain_op_read_flag("dtb_gain_contract", f, s);
    if (int* f = noalloc_flag(dev)) {
        const int rc2 = gain_op_read_flag("dtb_gain_contract_noalloc", f, s);
        if (rc == DTB_OK) rc = rc2;
    }
    if (rc == DTB_OK && cudaStreamSynchronize(s) != cudaSuccess) {
        set_error("dtb_gain_contract_status: stream synchronisation failed");
        return DTB_ECUDA;
    }
    return rc;
}

extern "C" int32_t dtb_selftest_gain_contract_timeout(int32_t noalloc, double limit_s, void* stream) {
    if (!(limit_s > 0 && limit_s <= 2.0)) {
        set_error("dtb_selftest_gain_contract_timeout: limit must be in (0, 2] s");
        return DTB_EINVAL;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("dtb_selftest_gain_contract_timeout: no current CUDA device");
        return DTB_ENODEV;
    }
    int* f = noalloc ? noalloc_flag(dev) : op_flag(dev);
    if (!f) {
        set_error("dtb_selftest_gain_contract_timeout: the entry has not run on this device yet");
        return DTB_ESTATE;
    }
    cudaError_t e = launch_bounded_wait_selftest((unsigned long long)(limit_s * 1e9), f,
                                                 reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_error(std::string("dtb_selftest_gain_contract_timeout: ") + cudaGetErrorString(e));
        return DTB_ECUDA;
    }
    return DTB_OK;
}
