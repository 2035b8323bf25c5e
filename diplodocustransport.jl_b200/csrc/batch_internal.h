// Internal declarations of the batched mixed-precision path (kernels_batch.cu, batch_api.cpp).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "dtb_internal.h"

namespace dtb {

constexpr int kMmaM = 128;  // rows of one UMMA tile (G rows)
constexpr int kMmaK = 64;   // K per stage: one 128-byte swizzle row of BF16

// Arguments of one gain-group GEMM: Y[i][r] = sum_k G[r][k] X[k][i] for the stacked output
// rows r of all gain blocks that share the input pair (in1, in2), with
// X[b * n2p + c][i] = (f_in1[b][i] * isig1[i]) * (f_in2[c][i] * isig2[i]).
struct GemmArgs {
    const unsigned char* gt;  // G tiles [m_tiles][T][hi, lo][128 rows x 128 B], pre-swizzled (see split_rows)
    int M;          // stacked rows of the group
    int N1;         // states of input species 1
    int n2;         // states of input species 2 (unpadded)
    int n_cb;       // 64-wide blocks of input species 2 (n2 padded to 64)
    int off1, off2; // state offsets of the two input species
    int tiles_per_split, n_splits, m_tiles, n_tiles;
    int splits_per_cb;  // > 0: every split lies inside one 64-wide input-2 block (K tiles cb-major)
    int Bcap;       // instances that exist (columns >= Bcap are zero in X)
    int Bst;        // row stride of the state matrix F[n_state][Bst]
    int n_space;    // space cells: column j of X is cell j / Bst of slot j % Bst
    int n_mom;      // states of one cell
    int Bpad;       // n_tiles * BN, instance stride of the partial rows
    const float* F;
    const float* isig1;  // [Bst] reciprocal power-of-two scale of species in1 per instance
    const float* isig2;
    float* partial;      // [n_splits][Bpad][M]
    int* err;
    const int* active_hi;  // device: 1 + the highest slot that still steps (columns past it are skipped)
    int ring_after_x0;     // 1: the G ring past its first tiles waits for the first X tile (tensor-bound
                           // groups, whose state loads must not queue behind the G stream); 0: the whole
                           // ring streams at once (HBM-bound groups)
};

cudaError_t launch_gain_gemm(int bn, const GemmArgs& a, cudaStream_t s);
// The CTA-pair variant (BN = 256, m_tiles even): grid m_tiles x n_tiles x n_splits CTAs in
// clusters of two. prepare_gain_gemm_pair raises the shared-memory limit and reports how many
// pairs fit on the device at once.
cudaError_t prepare_gain_gemm_pair(int* max_pairs);
cudaError_t launch_gain_gemm_pair(const GemmArgs& a, cudaStream_t s);

// Bytes of one K tile of one m tile of G: hi and lo halves of 128 rows x 64 BF16.
constexpr int kGTileBytes = 2 * kMmaM * kMmaK * 2;
int gain_gemm_smem_bytes(int bn);
cudaError_t prepare_gain_gemm(int bn);

// K chunks of loss / emission tile products one fast epilogue tile may run (more: direct path).
constexpr int kRowsMaxJobs = 32;
constexpr int kRowsChunk = 128;

// One K chunk of an epilogue tile product: kRowsChunk columns of a row-major operand (loss or
// emission rows, stored as BF16 hi and lo halves of the row-scaled values) against the same state
// rows of the tile's instances. Built on the host per 32-row tile.
struct RowJob {
    const __nv_bfloat16* TL;  // loss operand (hi half) at the tile's first row, column 0, or null;
                              // the lo half is ops.loss_lo elements further
    const __nv_bfloat16* TE;  // emission operand likewise (lo half ops.emi_lo further), or null
                              // (loss and emission over the same state rows share one job and
                              // one staged state chunk)
    int ldl, lde;     // operand row pitches (multiples of 8)
    int col0;         // state row of operand column 0
    int nc;           // operand columns
    int c0;           // first column of the chunk
    int pad;
};

// Per-row operands of the batched Euler epilogue.
struct MixedRowOps {
    int n_mom, Bcap, n_species;  // Bcap: slots in the state matrix (a multiple of 4), its row stride
    int n_state, n_space;        // rows of the state matrix = n_space cells of n_mom states
    const float* vol_cell;       // per cell: Vol (SteppingMethods.jl:380)
    const unsigned char* bin_on; // per cell: the binary term applies (BinM.Domain); null = every cell
    int sp_off[DTB_MAX_SPECIES + 1];
    int ell_w;
    const float* ell_val;
    const int* ell_col;
    const int* emi_rptr;
    const int* emi_piece;
    const long long* emi_data_off;
    const int* emi_ld;
    const int* emi_row0;
    const int* emi_col0;
    const int* emi_ncols;
    // E rows as BF16 hi halves of E[a][c] / emi_rscale[a], each row padded with zeros to emi_ld
    // (a multiple of 8); the lo halves (the BF16 rounding of the remainder) emi_lo elements further
    const __nv_bfloat16* emi_data;
    long long emi_lo;
    const float* emi_rscale;         // [n_state] power-of-two scale of each state row's emission
    int loss_ptr[DTB_MAX_SPECIES + 1];
    const long long* loss_data_off;
    const int* loss_ld;
    const int* loss_col_off;
    const int* loss_ncols;
    // loss rows likewise: hi halves of L[a][c] / loss_rscale[a], lo halves loss_lo elements further
    const __nv_bfloat16* loss_data;
    long long loss_lo;
    const float* loss_rscale;        // [n_mom] power-of-two scale of each momentum row's loss blocks
    // gain: for a row of species s, entries [gain_ptr[s], gain_ptr[s+1]) give (group, row offset)
    int gain_ptr[DTB_MAX_SPECIES + 1];
    int gain_grp[64];
    int gain_roff[64];
    // split-K partial sums of each gain group's GEMM: partial[split][column][M]; the epilogue sums
    // the splits in order and scales back by row_scale[r] * sig1[slot] * sig2[slot]
    const float* grp_partial[16];
    long long grp_stride[16];     // Bpad * M: elements between splits
    int grp_nsplit[16];
    int grp_M[16];
    const float* grp_rscale[16];
    const float* grp_sig1[16];    // [Bcap] power-of-two scale of input 1 per slot
    const float* grp_sig2[16];
    const unsigned char* tile_fast;  // per 32-row tile: loss/emission as shared-memory tile products
    const RowJob* jobs;              // [tile][kRowsMaxJobs] product chunks of the fast tiles
    const int* njobs;                // [tile]
    const float* invAp;
    const float* inj;
    double thr;
    int has_bin, has_emi;
    const double* dt_scale;          // [Bcap]
    const long long* stop_step;      // [Bcap]: the slot steps while gstep < stop_step
    unsigned long long* min_ratio;   // [Bcap] ordered encoding of min(df / f) over the run
    int* nonfinite;                  // [Bcap]
};

cudaError_t launch_mixed_rows(const MixedRowOps& ops, const float* F_in, const float* C_in, float* F_out,
                              float* C_out, const unsigned long long* gstep, int kpos, cudaStream_t s);
cudaError_t launch_advance_step(unsigned long long* gstep, int n, cudaStream_t s);

// Byte layout of one admission record (n states, ns species): f and compensation columns, the
// species scales and their reciprocals, dt / dt0 and the stop step; the record is staged in
// pinned memory, copied in one piece and scattered by admit_slot_kernel.
struct AdmitRecord {
    size_t f, c, sig, isig, dt, stop, bytes;
};
__host__ __device__ inline AdmitRecord admit_record(int n, int ns) {
    AdmitRecord r;
    r.f = 0;
    r.c = r.f + 4 * (size_t)n;
    r.sig = r.c + 4 * (size_t)n;
    r.isig = r.sig + 4 * (size_t)ns;
    r.dt = (r.isig + 4 * (size_t)ns + 7) / 8 * 8;
    r.stop = r.dt + 8;
    r.bytes = (r.stop + 8 + 255) / 256 * 256;
    return r;
}
cudaError_t launch_admit_slot(const unsigned char* rec, int n, int ns, int slot, int Bst, float* F, float* C, float* sig,
                              float* isig, double* dt_scale, long long* stop, unsigned long long* min_ratio,
                              int* nonfinite, unsigned long long inf_enc, cudaStream_t s);
cudaError_t launch_pack_f(const double* io, int Buser, int n, int Bcap, float* F, float* C, cudaStream_t s);
cudaError_t launch_unpack_f(const float* F, const float* C, int Buser, int n, int Bcap, double* io, cudaStream_t s);
int mixed_rows_tile_rows();
cudaError_t prepare_mixed_rows();

cudaError_t launch_batch_moments(const float* F, const float* C, int Bcap, const int* sp_off, int n_species,
                                 int n_mom, int n_space, const double* w, double* out, cudaStream_t s);

cudaError_t launch_split_rows(const float* src, long long rows, int row0, int n1, int n2, int n_cb,
                              unsigned char* gt, float* row_scale, cudaStream_t s);

}  // namespace dtb
