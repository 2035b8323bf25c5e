// Kernel-level entry for one gain block held in the caller's device memory:
//   out[a] = sum_b f1[b] sum_c G[a][b][c] f2[c]
// i.e. the two products of update_Big_Bin! (SteppingMethods.jl:372-373) restricted to one
// (output species, input-1 species, input-2 species) block, without the context API.
// It runs the same gain_stream kernel as the stepping path, followed by a per-row sum of the
// per-unit partials.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

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

int gain_op_plan(int64_t n_out, int64_t n1, int64_t n2, int esz, int num_sms, int bps, std::vector<GainUnit>& units,
                 int& splits) {
    const int64_t row_b = n2 * esz;
    if (n2 <= 0 || n2 % 8 != 0 || row_b > kGainTileBytes) {
        set_error("gain op: n2 must be a positive multiple of 8 with n2 * element size <= 16384 bytes");
        return DTB_EINVAL;
    }
    if (n_out <= 0 || n1 <= 0) {
        set_error("gain op: n_out and n1 must be positive");
        return DTB_EINVAL;
    }
    const double tot = (double)n_out * n1 * n2 * esz;
    const double target =
        std::min(256.0 * 1024, std::max((double)kGainTileBytes, tot / ((double)num_sms * std::max(1, bps) * 8)));
    const int tile_b = (int)std::max<int64_t>(1, std::min<int64_t>(n1, kGainTileBytes / row_b));
    const int64_t nb = std::max<int64_t>(tile_b, (int64_t)(target / row_b) / tile_b * tile_b);
    splits = (int)((n1 + nb - 1) / nb);
    units.clear();
    units.reserve((size_t)(n_out * splits));
    const int64_t offp1 = (n1 + 7) / 8 * 8;
    for (int64_t a = 0; a < n_out; ++a)
        for (int64_t b0 = 0; b0 < n1; b0 += nb) {
            GainUnit u;
            u.g_off = (a * n1 + b0) * n2;
            u.b_off = (int)b0;
            u.c_off = (int)offp1;
            u.nb = (int)std::min(nb, n1 - b0);
            u.n2p = (int)n2;
            u.tile_b = tile_b;
            u.row = (int)a;
            units.push_back(u);
        }
    return DTB_OK;
}

// Runs the contraction with scratch at `scratch` (units, then partials, then the f1|f2 vector).
int gain_op_run(int32_t dtype, const void* G, int64_t n_out, int64_t n1, int64_t n2, const void* f1, const void* f2,
                double* out, const std::vector<GainUnit>& units, int splits, unsigned char* scratch,
                int* err, cudaStream_t s) {
    const int esz = dtype == DTB_DTYPE_F64 ? 8 : 4;
    const int n_units = (int)units.size();
    const size_t units_bytes = ((size_t)n_units * sizeof(GainUnit) + 255) / 256 * 256;
    const size_t part_bytes = ((size_t)n_units * sizeof(double) + 255) / 256 * 256;
    GainUnit* d_units = reinterpret_cast<GainUnit*>(scratch);
    double* d_part = reinterpret_cast<double*>(scratch + units_bytes);
    unsigned char* d_f = scratch + units_bytes + part_bytes;
    const int64_t offp1 = (n1 + 7) / 8 * 8;
    cudaError_t e = cudaMemcpyAsync(d_units, units.data(), (size_t)n_units * sizeof(GainUnit), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_f, f1, (size_t)n1 * esz, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_f + n1 * esz, f2, (size_t)n2 * esz, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) {
        set_error(std::string("gain op: copy to scratch failed: ") + cudaGetErrorString(e));
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
    if (e == cudaSuccess) e = launch_row_sums(d_part, (int)n_out, splits, out, s);
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
}  // namespace

extern "C" int32_t dtb_gain_contract(int32_t dtype, const void* G, int64_t n_out, int64_t n1, int64_t n2,
                                     const void* f1, const void* f2, double* out, void* stream) {
    if (!G || !f1 || !f2 || !out) {
        set_error("dtb_gain_contract: null argument");
        return DTB_EINVAL;
    }
    if (dtype != DTB_DTYPE_F64 && dtype != DTB_DTYPE_F32) {
        set_error("dtb_gain_contract: bad dtype");
        return DTB_EINVAL;
    }
    const int esz = dtype == DTB_DTYPE_F64 ? 8 : 4;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("dtb_gain_contract: no current CUDA device");
        return DTB_ENODEV;
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    std::vector<GainUnit> units;
    int splits = 0;
    int rc = gain_op_plan(n_out, n1, n2, esz, sms, gain_stream_blocks_per_sm(esz, (int)((n1 + 7) / 8 * 8 + n2)), units,
                          splits);
    if (rc != DTB_OK) return rc;
    const size_t need = gain_op_scratch_bytes((int64_t)units.size(), n1, n2, esz);
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
    if (!sc.err) {
        if (cudaMalloc(&sc.err, sizeof(int)) != cudaSuccess || cudaMemsetAsync(sc.err, 0, sizeof(int), s) != cudaSuccess) {
            set_error("dtb_gain_contract: error-flag allocation failed");
            return DTB_ENOMEM;
        }
    }
    return gain_op_run(dtype, G, n_out, n1, n2, f1, f2, out, units, splits, sc.p, sc.err, s);
}
