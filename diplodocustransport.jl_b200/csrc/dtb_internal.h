// Internal declarations shared by the libdtb.so translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/dtb.h"

namespace dtb {

// Error flags a kernel may raise (bitwise OR into a device int).
enum : int {
    KERR_TIMEOUT_FULL = 1,   // consumer gave up waiting for a staged tile
    KERR_TIMEOUT_EMPTY = 2,  // producer gave up waiting for a free stage
    KERR_TIMEOUT_DRAIN = 4,  // producer gave up waiting for its own copies at exit
    KERR_BAD_UNIT = 8,       // a work unit failed its bounds check
    KERR_TMEM = 16,          // tensor-memory allocation failed
};

// Bound of every device-side spin wait, in nanoseconds of %globaltimer.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

// One gain work unit: output row `row` of one gain block over b-rows [b0, b0 + nb).
// g_off is the element offset of G[row][b0][0] in the concatenated block storage.
struct GainUnit {
    long long g_off;
    int b_off;    // padded smem offset of f_in1[b0]
    int c_off;    // padded smem offset of f_in2[0]
    int nb;       // b-rows in the unit
    int n2p;      // padded length of a b-row (multiple of 8)
    int tile_b;   // b-rows per staged tile
    int row;      // output state row (momentum index within a cell)
};
static_assert(sizeof(GainUnit) == 32, "GainUnit layout");

struct StepDiagDev {
    double cr[4];
    double sum_df;
    double sum_f;
    int finite;
    int pad;
};
static_assert(sizeof(StepDiagDev) == sizeof(dtb_step_diag), "diag layout");

// Per-row operand tables of the fused row kernel.
template <typename T>
struct RowOps {
    int n_mom, n_state, n_space;
    int n_species;
    int sp_off[DTB_MAX_SPECIES + 1];   // unpadded species offsets within a cell
    int sp_offp[DTB_MAX_SPECIES + 1];  // padded offsets (multiples of 8) used by the gain kernel
    // flux, banded ELL with width ell_w (multiple of 4), one row of ell_w slots per state;
    // unused slots have column -1
    int ell_w;
    const T* ell_val;
    const int* ell_col;
    // emission: per state row, list of pieces [emi_rptr[i], emi_rptr[i+1])
    const int* emi_rptr;
    const int* emi_piece;                  // piece index
    const long long* emi_data_off;         // per piece: element offset of its first row
    const int* emi_ld;                     // per piece: padded row length (multiple of 4)
    const int* emi_row0;                   // per piece: first global row
    const int* emi_col0;                   // per piece: first global column
    const int* emi_ncols;                  // per piece: columns
    const T* emi_data;
    // loss: per species, list of blocks [loss_ptr[s], loss_ptr[s+1])
    int loss_ptr[DTB_MAX_SPECIES + 1];
    const long long* loss_data_off;        // per block: element offset
    const int* loss_ld;                    // per block: padded row length
    const int* loss_col_off;               // per block: unpadded offset of the other species
    const int* loss_ncols;                 // per block
    const T* loss_data;
    // gain partials: units of row a are [unit_ptr[a], unit_ptr[a+1])
    const int* unit_ptr;
    int n_units;
    const double* partial;                 // [n_space][n_units]
    const unsigned char* bin_on;           // per cell: binary term applied (BinM.Domain); null = all
    // vectors
    const T* invAp;
    const T* inj;
    const T* vol;
    double thr;                            // clamp threshold in the state precision
    int has_bin, has_emi;
    // ForwardSymplecticEuler (SteppingMethods.jl:120-243): mode 1 is its momentum pass, which
    // writes f_Momentum (clamped at thr_mom) and df_Momentum; the space pass uses the X flux
    int mode;
    T* dfm_out;
    double thr_mom, thr_space;
    int x_ell_w;
    const T* x_ell_val;
    const int* x_ell_col;
};

// Launch helpers (kernels_plain.cu).
template <typename T>
cudaError_t launch_gain_stream(const T* G, const GainUnit* units, int n_units, const T* f,
                               int n_mom, const int* sp_offp_dev, int n_species, int f_smem_len,
                               double* partial, int n_space, int grid_x, int* err, cudaStream_t s,
                               const int* cell_list = nullptr, bool pdl = false);

// Fields of one row block's diagnostics record: min cr, cr_bin, cr_emi, cr_flux, sum df, sum f.
constexpr int kStepRecFields = 6;

// One step's rows. The step is number *ctr + kpos of the dt sequence (the counter advances
// only in launch_step_diag); each row block writes its diagnostics record to
// rec[blockIdx][kStepRecFields] (rec: the step's slot of the record buffer). pdl: launch as a
// programmatic dependent of the previous kernel, which must then be the step's gain kernel (the
// rows read the state before their dependency wait).
template <typename T>
cudaError_t launch_euler_rows(const RowOps<T>& ops, const T* f_in, T* f_out, double dt_imm,
                              const double* dt_arr, const unsigned long long* ctr, int kpos, int verbose,
                              double* rec, bool pdl, cudaStream_t s);
int euler_rows_blocks(int n_state);

// The diagnostics of steps *ctr .. *ctr + n_steps - 1: block k reduces step k's row-block
// records (slot k of blk_red, n_blocks records of kStepRecFields each) into
// hist[(*ctr + k) % hist_cap]; the last block to finish advances *ctr by n_steps. sympl: the
// records are the symplectic space pass's (no per-term Crs, no finite check).
cudaError_t launch_step_diag(const double* blk_red, int n_blocks, int n_steps, unsigned long long* ctr,
                             StepDiagDev* hist, long long hist_cap, int verbose, int has_bin, int has_emi, int sympl,
                             unsigned* ticket, cudaStream_t s);

// The symplectic space pass of a step numbered like launch_euler_rows'; its row blocks write
// records in the same layout (the whole-step Cr and the f sum only).
template <typename T>
cudaError_t launch_sympl_space(const RowOps<T>& ops, const T* f_old, const T* fm, const T* dfm, T* f_out,
                               double dt_imm, const double* dt_arr, const unsigned long long* ctr, int kpos,
                               double* rec, cudaStream_t s);

template <typename Tin, typename Tout>
cudaError_t launch_pad_rows(const Tin* src, long long rows, int n, Tout* dst, int np, cudaStream_t s);

cudaError_t launch_moments_f64(const double* f, int n_mom, int n_space, const int* sp_off,
                               int n_species, const double* w, double* out, cudaStream_t s);
cudaError_t launch_moments_f32(const float* f, int n_mom, int n_space, const int* sp_off,
                               int n_species, const double* w, double* out, cudaStream_t s);

cudaError_t launch_bounded_wait_selftest(unsigned long long limit_ns, int* err, cudaStream_t s);

int gain_stream_smem_bytes(int elem_size, int f_smem_len);
int gain_stream_blocks_per_sm(int elem_size, int f_smem_len);
constexpr int kGainTileBytes = 16384;
constexpr int kGainStages = 4;
constexpr int kGainConsumerWarps = 8;
constexpr int kRowsWarps = 8;

void set_error(const std::string& msg);

// Kernel-level gain contraction of one block (gain_op.cu).
cudaError_t launch_row_sums(const double* partial, int n_rows, int splits, double* out, cudaStream_t s);
}  // namespace dtb
namespace dtb {
// Work split of one kernel-level gain contraction: n_out rows x `splits` b-ranges of `nb`
// b-rows each, staged `tile_b` b-rows per tile.
struct GainOpPlan {
    int64_t n_units;
    int splits;
    int64_t nb;
    int tile_b;
};
int gain_op_plan(int64_t n_out, int64_t n1, int64_t n2, int esz, int num_sms, int bps, GainOpPlan& plan);
int gain_op_run(int32_t dtype, const void* G, int64_t n_out, int64_t n1, int64_t n2, const void* f1, const void* f2,
                double* out, const GainOpPlan& plan, unsigned char* scratch, int* err, cudaStream_t s);
size_t gain_op_scratch_bytes(int64_t n_units, int64_t n1, int64_t n2, int esz);
// Common argument checks of the kernel-level entries (null pointers, dtype, alignment).
int gain_op_check_args(const char* who, int32_t dtype, const void* G, const void* f1, const void* f2,
                       const double* out);
// Reads (synchronising `s`) and clears a kernel-level entry's device error flag.
int gain_op_read_flag(const char* who, int* err, cudaStream_t s);

}  // namespace dtb
