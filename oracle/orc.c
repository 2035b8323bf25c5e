/*
 * Oracle for the explicit (forward) Euler step of DiplodocusTransport.jl.
 *
 * TEST INFRASTRUCTURE ONLY. This file is a plain-C FP64 restatement of the
 * reference's algorithm, used by the tests, by the smoke check and by the
 * CPU-baseline leg of bench.py to check results. Nothing in the product library
 * links, calls or falls back to it.
 *
 * Parity status: the reference (Julia) cannot run without a Julia toolchain and its
 * own test suite is empty (test/runtests.jl:4-6), so no reference-produced
 * vectors exist. This restatement is pinned instead against hand-derived
 * known-answer vectors and a literal pure-Python transliteration of the cited
 * Julia lines (tests/golden/make_golden.py); parity against a run of the
 * reference itself is unpinned.
 *
 * Followed lines (paths relative to the reference project):
 *   src/SteppingMethods.jl:12-107   ForwardEuler functor: df assembly, scaling,
 *                                    CFL diagnostics, update and clamps
 *   src/SteppingMethods.jl:332-397  update_Big_Bin!: S = reshape(M_Bin f), df = Vol S f
 *   src/SteppingMethods.jl:120-243  ForwardSymplecticEuler functor
 *   src/SteppingStructs.jl:55,60    invAp = 1 ./ Ap, F = X + P
 *   src/Collisions/BuildBinaryMatrices.jl:181-196,261-276  M_Bin index map
 *                                    (blocked form == reference layout)
 *   src/DistributionMoments.jl:33,145,162  number and energy moments
 *
 * Julia semantics reproduced exactly:
 *   - `x * b::Bool` is ifelse(b, x, copysign(0, x)) (a strong zero: NaN*false
 *     and Inf*false give a signed zero, never NaN);
 *   - the clamp literal 1f-10 is a Float32 promoted to Float64 when compared
 *     with a Float64 state, i.e. the threshold is (double)1e-10f;
 *   - `mapreduce(x -> isnan(x) ? Inf : x, min, v)` with Julia's min, which
 *     orders -0.0 below +0.0 and propagates nothing else special.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2

/* Julia `x * (cond)` with a Bool. */
static inline double jl_mul_bool(double x, int b) { return b ? x : copysign(0.0, x); }

/* Julia min for Float64 (NaN already mapped to Inf by the caller). */
static inline double jl_min(double a, double b) {
    if (a < b) return a;
    if (b < a) return b;
    /* equal, or +-0: Julia's min returns -0.0 when either is -0.0 */
    if (signbit(a)) return a;
    return b;
}

static inline double nan_to_inf(double x) { return isnan(x) ? INFINITY : x; }

/* Julia `@. f = f*(f>=thr)` then `@. f = f*(f!=Inf)` (SteppingMethods.jl:99,101). */
static inline double clamp_state(double f, double thr) {
    f = jl_mul_bool(f, f >= thr);
    f = jl_mul_bool(f, f != INFINITY);
    return f;
}

double orc_clamp(double f, double thr) { return clamp_state(f, thr); }
double orc_threshold_f64(void) { return (double)1e-10f; }

/* ---- CSC sparse product, SparseArrays' column-ordered accumulation ---- */
static void csc_mul(int64_t n, const int64_t* colptr, const int64_t* rowval,
                    const double* nzval, int base, const double* x, double* y) {
    memset(y, 0, sizeof(double) * (size_t)n);
    if (!colptr) return;
    for (int64_t j = 0; j < n; ++j) {
        double xj = x[j];
        for (int64_t p = colptr[j] - base; p < colptr[j + 1] - base; ++p)
            y[rowval[p] - base] += nzval[p] * xj;
    }
}

/* Dense column-major GEMV y = A x, A is m x n (leading dim m). */
static void gemv_colmajor(int64_t m, int64_t n, const double* A, const double* x, double* y) {
#pragma omp parallel
    {
#ifdef _OPENMP
        int nt = omp_get_num_threads(), t = omp_get_thread_num();
#else
        int nt = 1, t = 0;
#endif
        int64_t chunk = (m + nt - 1) / nt;
        int64_t r0 = t * chunk, r1 = r0 + chunk < m ? r0 + chunk : m;
        for (int64_t r = r0; r < r1; ++r) y[r] = 0.0;
        for (int64_t k = 0; k < n; ++k) {
            const double* col = A + (size_t)k * (size_t)m;
            double xk = x[k];
            for (int64_t r = r0; r < r1; ++r) y[r] += col[r] * xk;
        }
    }
}

/*
 * Diagnostics written by the step functions (diag[0..7]):
 *   0 Cr, 1 Cr_Bin, 2 Cr_Emi, 3 Cr_Flux (SteppingMethods.jl:52-94),
 *   4 finite flag = isfinite(sum(df)) (:48), 5 sum(df), 6 sum(f_old)
 */
static void cfl_diag(int64_t n, int verbose, int has_bin, int has_emi,
                     const double* f, const double* df, const double* df_bin,
                     const double* df_emi, const double* df_flux, double* diag) {
    double sdf = 0.0, sf = 0.0;
    for (int64_t i = 0; i < n; ++i) { sdf += df[i]; sf += f[i]; }
    diag[0] = diag[1] = diag[2] = diag[3] = 0.0;
    diag[4] = isfinite(sdf) ? 1.0 : 0.0;
    diag[5] = sdf;
    diag[6] = sf;
    if (!(verbose == 1 || verbose == 2 || verbose == 3)) return;
    if (sf == 0.0) return;
    if (verbose == 3) {
        if (has_bin) {
            double m = INFINITY;
            for (int64_t i = 0; i < n; ++i) m = jl_min(m, nan_to_inf(df_bin[i] / f[i]));
            diag[1] = -m;
        }
        if (has_emi) {
            double m = INFINITY;
            for (int64_t i = 0; i < n; ++i) m = jl_min(m, nan_to_inf(df_emi[i] / f[i]));
            diag[2] = -m;
        }
        double m = INFINITY;
        for (int64_t i = 0; i < n; ++i) m = jl_min(m, nan_to_inf(-df_flux[i] / f[i]));
        diag[3] = -m;
    }
    double m = INFINITY;
    for (int64_t i = 0; i < n; ++i) m = jl_min(m, nan_to_inf(df[i] / f[i]));
    diag[0] = -m;
}

/* update_Big_Bin! skips a space cell (SteppingMethods.jl:369) unless the binary domain is
 * `nothing` (dom == NULL), the cell's off_space is in the domain, or the cell's f has no
 * nonzero entry (findfirst(!iszero, fView) === nothing; NaN counts as nonzero). A skipped
 * cell keeps df_Bin from its last evaluation, which for a finite M_Bin is the all-zero f
 * result: zeros. dom: one byte per cell, nonzero = in the domain. */
static int bin_cell_on(const uint8_t* dom, int64_t cell, const double* fv, int64_t n_mom) {
    if (!dom || dom[cell]) return 1;
    for (int64_t k = 0; k < n_mom; ++k)
        if (fv[k] != 0.0) return 0;
    return 1;
}

/*
 * One ForwardEuler step in the reference layout (SteppingMethods.jl:12-107).
 *   M_Bin: (n_mom^2) x n_mom column-major, or NULL (no binary interactions)
 *   M_Emi: n x n column-major, or NULL (no emission), n = n_mom * n_space
 *   F = X + P as CSC (colptr n+1, rowval/nzval), indices with base `base`
 *   invAp, inj: length n; Vol: length n_space
 *   thr: clamp threshold ((double)1e-10f for a Float64 state)
 *   f: state, updated in place; diag: 8 doubles (see cfl_diag)
 *   df_out: optional, receives the scaled df (length n)
 *   bin_dom: NULL (Bin_Domain === nothing) or one byte per cell (see bin_cell_on)
 */
int orc_step_ref(int64_t n_mom, int64_t n_space, const double* M_Bin, const double* M_Emi,
                 const int64_t* colptr, const int64_t* rowval, const double* nzval, int base,
                 const double* invAp, const double* Vol, const double* inj, double dt_scale,
                 double thr, int verbose, double* f, double* diag, double* df_out, const uint8_t* bin_dom) {
    int64_t n = n_mom * n_space;
    double* buf = (double*)malloc(sizeof(double) * (size_t)(4 * n + n_mom * n_mom));
    if (!buf) return ORC_ENOMEM;
    double *df = buf, *df_flux = buf + n, *df_emi = buf + 2 * n, *df_bin = buf + 3 * n;
    double* S = buf + 4 * n; /* M_Bin_Mul_Step, n_mom x n_mom column-major */

    /* :31-32 */
    csc_mul(n, colptr, rowval, nzval, base, f, df_flux);
    for (int64_t i = 0; i < n; ++i) df[i] = -df_flux[i];
    /* :35-38 */
    memset(df_emi, 0, sizeof(double) * (size_t)n);
    if (M_Emi) {
        gemv_colmajor(n, n, M_Emi, f, df_emi);
        for (int64_t i = 0; i < n; ++i) df[i] += df_emi[i];
    }
    /* :41-44 -> update_Big_Bin! :360-386 */
    memset(df_bin, 0, sizeof(double) * (size_t)n);
    if (M_Bin) {
        for (int64_t cell = 0; cell < n_space; ++cell) {
            const double* fv = f + cell * n_mom;
            double* dv = df_bin + cell * n_mom;
            if (!bin_cell_on(bin_dom, cell, fv, n_mom)) continue; /* :369 */
            gemv_colmajor(n_mom * n_mom, n_mom, M_Bin, fv, S); /* :372 */
            gemv_colmajor(n_mom, n_mom, S, fv, dv);             /* :373 */
            for (int64_t a = 0; a < n_mom; ++a) dv[a] *= Vol[cell]; /* :380 */
        }
        for (int64_t i = 0; i < n; ++i) df[i] += df_bin[i];
    }
    /* :46 */
    for (int64_t i = 0; i < n; ++i) df[i] *= invAp[i] * dt_scale;
    /* :48-94 */
    cfl_diag(n, verbose, M_Bin != NULL, M_Emi != NULL, f, df, df_bin, df_emi, df_flux, diag);
    /* :97-101 */
    for (int64_t i = 0; i < n; ++i) {
        double v = f[i] + (df[i] + inj[i] * dt_scale);
        f[i] = clamp_state(v, thr);
    }
    if (df_out) memcpy(df_out, df, sizeof(double) * (size_t)n);
    free(buf);
    return ORC_OK;
}

/* ---------------- blocked form ----------------
 * Gain block: df[a] += sum_{b in in1, c in in2} G[a][b][c] f_b f_c,
 *   G row-major [N_out][N_in1][N_in2] (c fastest).
 * Loss block: df[a] -= f_a * sum_{c in other} L[a][c] f_c, L row-major [N_sp][N_other].
 * Both act per space cell on the cell's momentum slice and are scaled by Vol[cell].
 * Emission blocks are dense row-major pieces of the global n x n M_Emi.
 */
typedef struct { int32_t out_sp, in1_sp, in2_sp, pad; const double* G; } orc_gain_t;
typedef struct { int32_t row_sp, col_sp; const double* L; } orc_loss_t;
typedef struct { int64_t row0, nrows, col0, ncols; const double* E; } orc_emi_t;

/* Gain contraction of one block for rows [r0, r1): out[a - r0] = sum_b f1[b] sum_c G f2[c]. */
void orc_gain_rows(const double* G, int64_t r0, int64_t r1, int64_t n1, int64_t n2,
                   const double* f1, const double* f2, double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t a = r0; a < r1; ++a) {
        const double* row = G + (size_t)a * (size_t)(n1 * n2);
        double acc = 0.0;
        for (int64_t b = 0; b < n1; ++b) {
            const double* g = row + b * n2;
            double s = 0.0;
            for (int64_t c = 0; c < n2; ++c) s += g[c] * f2[c];
            acc += f1[b] * s;
        }
        out[a - r0] = acc;
    }
}

/* df_bin for one cell in the blocked form (gain - loss), not yet scaled by Vol. */
static void blocked_bin_cell(int32_t n_species, const int64_t* sp_size, const int64_t* sp_off,
                             int n_gain, const orc_gain_t* gains, int n_loss,
                             const orc_loss_t* losses, const double* fv, double* out, int64_t n_mom) {
    double* gain = (double*)calloc((size_t)n_mom, sizeof(double));
    double* loss = (double*)calloc((size_t)n_mom, sizeof(double));
    for (int g = 0; g < n_gain; ++g) {
        const orc_gain_t* B = &gains[g];
        int64_t no = sp_size[B->out_sp], n1 = sp_size[B->in1_sp], n2 = sp_size[B->in2_sp];
        double* tmp = (double*)malloc(sizeof(double) * (size_t)no);
        orc_gain_rows(B->G, 0, no, n1, n2, fv + sp_off[B->in1_sp], fv + sp_off[B->in2_sp], tmp);
        for (int64_t a = 0; a < no; ++a) gain[sp_off[B->out_sp] + a] += tmp[a];
        free(tmp);
    }
    for (int l = 0; l < n_loss; ++l) {
        const orc_loss_t* B = &losses[l];
        int64_t nr = sp_size[B->row_sp], nc = sp_size[B->col_sp];
        const double* fc = fv + sp_off[B->col_sp];
        for (int64_t a = 0; a < nr; ++a) {
            const double* row = B->L + a * nc;
            double s = 0.0;
            for (int64_t c = 0; c < nc; ++c) s += row[c] * fc[c];
            loss[sp_off[B->row_sp] + a] += s;
        }
    }
    for (int64_t a = 0; a < n_mom; ++a) out[a] = gain[a] - fv[a] * loss[a];
    free(gain);
    free(loss);
    (void)n_species;
}

/*
 * One ForwardEuler step with the binary and emission operators in blocked form.
 * Same semantics as orc_step_ref; used for sizes whose reference layout does
 * not fit in host memory.
 */
int orc_step_blocked(int32_t n_species, const int64_t* sp_size, int64_t n_space,
                     int n_gain, const orc_gain_t* gains, int n_loss, const orc_loss_t* losses,
                     int n_emi, const orc_emi_t* emis,
                     const int64_t* colptr, const int64_t* rowval, const double* nzval, int base,
                     const double* invAp, const double* Vol, const double* inj, double dt_scale,
                     double thr, int verbose, double* f, double* diag, double* df_out,
                     const uint8_t* bin_dom) {
    int64_t sp_off[64];
    if (n_species > 64) return ORC_EINVAL;
    int64_t n_mom = 0;
    for (int s = 0; s < n_species; ++s) { sp_off[s] = n_mom; n_mom += sp_size[s]; }
    int64_t n = n_mom * n_space;
    double* buf = (double*)malloc(sizeof(double) * (size_t)(4 * n));
    if (!buf) return ORC_ENOMEM;
    double *df = buf, *df_flux = buf + n, *df_emi = buf + 2 * n, *df_bin = buf + 3 * n;

    csc_mul(n, colptr, rowval, nzval, base, f, df_flux);
    for (int64_t i = 0; i < n; ++i) df[i] = -df_flux[i];
    memset(df_emi, 0, sizeof(double) * (size_t)n);
    if (n_emi > 0) {
        for (int e = 0; e < n_emi; ++e) {
            const orc_emi_t* B = &emis[e];
            for (int64_t r = 0; r < B->nrows; ++r) {
                const double* row = B->E + r * B->ncols;
                double s = 0.0;
                for (int64_t c = 0; c < B->ncols; ++c) s += row[c] * f[B->col0 + c];
                df_emi[B->row0 + r] += s;
            }
        }
        for (int64_t i = 0; i < n; ++i) df[i] += df_emi[i];
    }
    memset(df_bin, 0, sizeof(double) * (size_t)n);
    int has_bin = (n_gain + n_loss) > 0;
    if (has_bin) {
        for (int64_t cell = 0; cell < n_space; ++cell) {
            if (!bin_cell_on(bin_dom, cell, f + cell * n_mom, n_mom)) continue;
            blocked_bin_cell(n_species, sp_size, sp_off, n_gain, gains, n_loss, losses,
                             f + cell * n_mom, df_bin + cell * n_mom, n_mom);
            for (int64_t a = 0; a < n_mom; ++a) df_bin[cell * n_mom + a] *= Vol[cell];
        }
        for (int64_t i = 0; i < n; ++i) df[i] += df_bin[i];
    }
    for (int64_t i = 0; i < n; ++i) df[i] *= invAp[i] * dt_scale;
    cfl_diag(n, verbose, has_bin, n_emi > 0, f, df, df_bin, df_emi, df_flux, diag);
    for (int64_t i = 0; i < n; ++i) {
        double v = f[i] + (df[i] + inj[i] * dt_scale);
        f[i] = clamp_state(v, thr);
    }
    if (df_out) memcpy(df_out, df, sizeof(double) * (size_t)n);
    free(buf);
    return ORC_OK;
}

/*
 * One ForwardSymplecticEuler step in the reference layout (SteppingMethods.jl:120-243).
 * X and P are separate CSC matrices. diag[0] = Cr of the whole step (:217-218).
 */
int orc_step_symplectic_ref(int64_t n_mom, int64_t n_space, const double* M_Bin, const double* M_Emi,
                            const int64_t* xcolptr, const int64_t* xrowval, const double* xnzval,
                            const int64_t* pcolptr, const int64_t* prowval, const double* pnzval,
                            int base, const double* invAp, const double* Vol, const double* inj,
                            double dt_scale, double thr_mom, double thr_space, int verbose,
                            double* f, double* diag, const uint8_t* bin_dom) {
    int64_t n = n_mom * n_space;
    double* buf = (double*)malloc(sizeof(double) * (size_t)(8 * n + n_mom * n_mom));
    if (!buf) return ORC_ENOMEM;
    double *dfm = buf, *dpf = buf + n, *demi = buf + 2 * n, *dbin = buf + 3 * n;
    double *fm = buf + 4 * n, *dxf = buf + 5 * n, *dsp = buf + 6 * n, *fs = buf + 7 * n;
    double* S = buf + 8 * n;
    /* :140-141 */
    csc_mul(n, pcolptr, prowval, pnzval, base, f, dpf);
    for (int64_t i = 0; i < n; ++i) dfm[i] = -dpf[i];
    memset(demi, 0, sizeof(double) * (size_t)n);
    if (M_Emi) { /* :144-147 */
        gemv_colmajor(n, n, M_Emi, f, demi);
        for (int64_t i = 0; i < n; ++i) dfm[i] += demi[i];
    }
    memset(dbin, 0, sizeof(double) * (size_t)n);
    if (M_Bin) { /* :150-153 */
        for (int64_t cell = 0; cell < n_space; ++cell) {
            const double* fv = f + cell * n_mom;
            double* dv = dbin + cell * n_mom;
            if (!bin_cell_on(bin_dom, cell, fv, n_mom)) continue;
            gemv_colmajor(n_mom * n_mom, n_mom, M_Bin, fv, S);
            gemv_colmajor(n_mom, n_mom, S, fv, dv);
            for (int64_t a = 0; a < n_mom; ++a) dv[a] *= Vol[cell];
        }
        for (int64_t i = 0; i < n; ++i) dfm[i] += dbin[i];
    }
    for (int64_t i = 0; i < n; ++i) dfm[i] *= invAp[i] * dt_scale;                 /* :155 */
    for (int64_t i = 0; i < n; ++i) fm[i] = jl_mul_bool(f[i] + dfm[i], f[i] + dfm[i] >= thr_mom); /* :158-160 */
    csc_mul(n, xcolptr, xrowval, xnzval, base, fm, dxf);                              /* :165 */
    for (int64_t i = 0; i < n; ++i) dsp[i] = -dxf[i] * invAp[i] * dt_scale;         /* :166 */
    for (int64_t i = 0; i < n; ++i) fs[i] = jl_mul_bool(fm[i] + dsp[i], fm[i] + dsp[i] >= thr_space); /* :169-171 */
    /* :175-220, Cr of the whole step */
    double sf = 0.0;
    for (int64_t i = 0; i < n; ++i) sf += f[i];
    diag[0] = 0.0;
    if ((verbose == 1 || verbose == 2 || verbose == 3) && sf != 0.0) {
        double m = INFINITY;
        for (int64_t i = 0; i < n; ++i) m = jl_min(m, nan_to_inf((dsp[i] + dfm[i]) / f[i]));
        diag[0] = -m;
    }
    /* :233-237; sign(x) of Julia: -1, 0 or 1 (signed zero kept), NaN -> NaN */
    for (int64_t i = 0; i < n; ++i) {
        double v = fs[i] + inj[i] * dt_scale;
        double sg = isnan(v) ? v : (v > 0 ? 1.0 : (v < 0 ? -1.0 : v));
        v = jl_mul_bool(v, v >= thr_space) * sg;
        v = jl_mul_bool(v, v != INFINITY);
        f[i] = v;
    }
    free(buf);
    return ORC_OK;
}

/* Per-species number and energy moments (DistributionMoments.jl:33,145,162) of one cell,
 * given per-state energy weights w (cell-averaged energy); FP64 sums in state order. */
void orc_moments(int32_t n_species, const int64_t* sp_size, const double* f, const double* w,
                 double* num, double* energy) {
    int64_t off = 0;
    for (int s = 0; s < n_species; ++s) {
        double a = 0.0, e = 0.0;
        for (int64_t i = 0; i < sp_size[s]; ++i) { a += f[off + i]; e += f[off + i] * w[off + i]; }
        num[s] = a;
        energy[s] = e;
        off += sp_size[s];
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
