// C ABI of libdtb.so: context, operator uploads and re-layout, stepping, Solve loop.
//
// The context plays the role of ForwardEulerStruct (SteppingStructs.jl:2-102) for the B200
// backend: it owns the operators in device memory and the device state. The functor
// (SteppingMethods.jl:12-107) is dtb_step; Solve (Solver.jl:1-64) is dtb_solve, which keeps
// the reference's host-side dt logic and replays captured CUDA graphs between save points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "ctx.h"

namespace dtb {
thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
}  // namespace dtb

using namespace dtb;

int commit_mixed(dtb_ctx* c);     // batch_api.cpp
void destroy_mixed(dtb_ctx* c);   // batch_api.cpp

extern "C" {

int32_t dtb_abi_version(void) { return DTB_ABI_VERSION; }

const char* dtb_last_error(void) { return dtb::g_err.c_str(); }

int32_t dtb_device_count(int32_t* n) {
    DTB_CHECK(n, DTB_EINVAL, "dtb_device_count: null output");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        *n = 0;
        set_error(std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
        return DTB_ENODEV;
    }
    *n = c;
    return DTB_OK;
}

}  // extern "C"

namespace dtb {
const char* profile_path() {
    static const char* p = [] {
        const char* e = std::getenv("DTB_PROFILE");
        return (e && *e) ? e : nullptr;
    }();
    return p;
}
}  // namespace dtb

// One JSON line per context: its shape, the steps it launched, its device bytes and, when
// per-launch timing was on, the gain kernel's average launch time.
static void write_profile(const dtb_ctx* c, const char* path) {
    static std::mutex mu;
    std::string js = "{\"precision\": " + std::to_string(c->prec) + ", \"n_state\": " + std::to_string(c->n_state) +
                     ", \"n_space\": " + std::to_string(c->n_space) + ", \"device\": " + std::to_string(c->device) +
                     ", \"steps_run\": " + std::to_string(c->steps_run) + ", \"device_bytes\": " +
                     std::to_string(c->dev_bytes) + ", \"gain_bytes_per_step\": " + std::to_string(c->gain_bytes);
    if (c->prec == DTB_MIXED) {
        js += ", " + batch_profile_json(c);
    } else if (c->prof_n > 0) {
        char b[64];
        std::snprintf(b, sizeof(b), "%.6g", c->prof_ms / (double)c->prof_n);
        js += std::string(", \"gain_kernel_avg_ms\": ") + b + ", \"gain_kernel_launches\": " + std::to_string(c->prof_n);
    }
    js += "}\n";
    std::lock_guard<std::mutex> lk(mu);
    if (FILE* f = std::fopen(path, "a")) {
        std::fputs(js.c_str(), f);
        std::fclose(f);
    }
}

extern "C" {

int32_t dtb_create(const dtb_dims* dims, const dtb_opts* opts, dtb_ctx** out) {
    DTB_CHECK(dims && opts && out, DTB_EINVAL, "dtb_create: null argument");
    *out = nullptr;
    DTB_CHECK(dims->n_species >= 1 && dims->n_species <= DTB_MAX_SPECIES, DTB_EINVAL,
              "dtb_create: n_species must be in [1, 16]");
    DTB_CHECK(dims->n_space >= 1, DTB_EINVAL, "dtb_create: n_space must be >= 1");
    DTB_CHECK(opts->precision == DTB_F64 || opts->precision == DTB_F32 || opts->precision == DTB_MIXED, DTB_EINVAL,
              "dtb_create: precision must be DTB_F64, DTB_F32 or DTB_MIXED");
    DTB_CHECK(opts->index_base == 0 || opts->index_base == 1, DTB_EINVAL, "dtb_create: index_base must be 0 or 1");
    DTB_CHECK(opts->precision == DTB_MIXED || opts->batch <= 1, DTB_EINVAL,
              "dtb_create: the plain method takes batch 1 (batched instances need DTB_MIXED)");
    DTB_CHECK(opts->precision != DTB_MIXED || (opts->batch >= 1 && opts->batch <= 65536), DTB_EINVAL,
              "dtb_create: a batched context needs 1 <= batch <= 65536");
    DTB_CHECK(std::isfinite(opts->dt0) && opts->dt0 > 0, DTB_EINVAL, "dtb_create: dt0 must be finite and > 0");
    // graph_steps also sizes the step-record buffer (graph_steps x rows / 8 x 48 B) and the
    // batched path's set of captured graphs (one per length 1..graph_steps)
    DTB_CHECK(opts->graph_steps >= 0 && opts->graph_steps <= kMaxGraphSteps, DTB_EINVAL,
              "dtb_create: graph_steps must be in [0, " + std::to_string(kMaxGraphSteps) + "]");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("dtb_create: no CUDA device available");
        return DTB_ENODEV;
    }
    DTB_CHECK(opts->device >= 0 && opts->device < ndev, DTB_EINVAL, "dtb_create: bad device ordinal");
    std::unique_ptr<dtb_ctx> c(new dtb_ctx());
    c->dims = *dims;
    c->opts = *opts;
    c->ns = dims->n_species;
    c->n_space = dims->n_space;
    c->prec = opts->precision;
    c->esz = c->prec == DTB_F64 ? 8 : 4;  // state element size (DTB_MIXED keeps f in FP32)
    c->device = opts->device;
    c->symplectic = (opts->flags & DTB_FLAG_SYMPLECTIC) != 0;
    DTB_CHECK(!c->symplectic || c->prec != DTB_MIXED, DTB_EINVAL,
              "dtb_create: the symplectic method is available for DTB_F64 / DTB_F32 contexts");
    c->off[0] = 0;
    c->offp[0] = 0;
    for (int s = 0; s < c->ns; ++s) {
        DTB_CHECK(dims->species_size[s] >= 1, DTB_EINVAL, "dtb_create: species_size must be >= 1");
        c->sz[s] = dims->species_size[s];
        c->off[s + 1] = c->off[s] + c->sz[s];
        c->offp[s + 1] = c->offp[s] + round_up(c->sz[s], 8);
    }
    c->n_mom = c->off[c->ns];
    c->n_state = c->n_mom * c->n_space;
    DTB_CHECK(c->n_state < (int64_t)1 << 30, DTB_EINVAL, "dtb_create: state vector too long");
    if (opts->graph_steps > 0) {
        c->graph_steps = (opts->graph_steps + 1) / 2 * 2;
    } else {
        // Default: 64 steps per graph, since a graph boundary costs a small grid about two thirds
        // of a step (config 0: 9.42 us per step with 16, 9.11 with 64), as long as the step
        // records of 64 steps take at most 8 MB (about 175,000 states); else 16.
        const int64_t rec64 = (int64_t)sizeof(double) * kStepRecFields * ((c->n_state + kRowsWarps - 1) / kRowsWarps) * 64;
        c->graph_steps = rec64 <= ((int64_t)8 << 20) ? 64 : 16;
    }
    DeviceGuard g(c->device);
    cudaDeviceProp prop;
    DTB_CUDA(cudaGetDeviceProperties(&prop, c->device));
    c->num_sms = prop.multiProcessorCount;
    if (opts->stream) {
        c->stream = reinterpret_cast<cudaStream_t>(opts->stream);
    } else {
        DTB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    *out = c.release();
    return DTB_OK;
}

int32_t dtb_destroy(dtb_ctx* c) {
    if (!c) return DTB_OK;
    DeviceGuard g(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (const char* path = profile_path()) write_profile(c, path);
    destroy_mixed(c);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
    c->free_all();
    if (c->pin_dt) cudaFreeHost(c->pin_dt);
    if (c->pin_hist) cudaFreeHost(c->pin_hist);
    if (c->pin_err) cudaFreeHost(c->pin_err);
    if (c->pin_f32) cudaFreeHost(c->pin_f32);
    if (c->pin_dt2) cudaFreeHost(c->pin_dt2);
    if (c->pin_hist2) cudaFreeHost(c->pin_hist2);
    if (c->save_pin) cudaFreeHost(c->save_pin);
    if (c->pipe_ready) {
        for (cudaEvent_t e : c->pipe_ev)
            if (e) cudaEventDestroy(e);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return DTB_OK;
}


static int add_csc(dtb_ctx* c, std::vector<int64_t>& R, std::vector<int64_t>& Cv, std::vector<double>& V, int64_t n,
                   const int64_t* colptr, const int64_t* rowval, const double* nzval) {
    DTB_CHECK(!c->committed, DTB_ESTATE, "dtb_add_flux_csc: operators already committed");
    DTB_CHECK(n == c->n_state, DTB_EINVAL, "dtb_add_flux_csc: n must equal the state length");
    DTB_CHECK(colptr, DTB_EINVAL, "dtb_add_flux_csc: null colptr");
    const int64_t base = c->opts.index_base;
    const int64_t nnz = colptr[n] - colptr[0];
    DTB_CHECK(colptr[0] == base && nnz >= 0, DTB_EINVAL, "dtb_add_flux_csc: colptr[0] must equal index_base");
    DTB_CHECK(nnz == 0 || (rowval && nzval), DTB_EINVAL, "dtb_add_flux_csc: null rowval/nzval");
    for (int64_t j = 0; j < n; ++j) {
        DTB_CHECK(colptr[j + 1] >= colptr[j], DTB_EINVAL, "dtb_add_flux_csc: colptr not monotone");
        for (int64_t p = colptr[j] - base; p < colptr[j + 1] - base; ++p) {
            const int64_t r = rowval[p] - base;
            DTB_CHECK(r >= 0 && r < n, DTB_EINVAL,
                      "dtb_add_flux_csc: row index out of range at entry " + std::to_string(p));
            R.push_back(r);
            Cv.push_back(j);
            V.push_back(nzval[p]);
        }
    }
    return DTB_OK;
}

int32_t dtb_add_flux_csc(dtb_ctx* c, int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_add_flux_csc: null context");
    DTB_CHECK(!c->symplectic, DTB_EINVAL,
              "dtb_add_flux_csc: the symplectic method keeps X and P apart; use dtb_add_flux_csc_part");
    return add_csc(c, c->flux_r, c->flux_c, c->flux_v, n, colptr, rowval, nzval);
}

int32_t dtb_add_flux_csc_part(dtb_ctx* c, int32_t part, int64_t n, const int64_t* colptr, const int64_t* rowval,
                              const double* nzval) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_add_flux_csc_part: null context");
    DTB_CHECK(part == DTB_FLUX_X || part == DTB_FLUX_P, DTB_EINVAL, "dtb_add_flux_csc_part: part must be X or P");
    if (c->symplectic && part == DTB_FLUX_X) return add_csc(c, c->xflux_r, c->xflux_c, c->xflux_v, n, colptr, rowval, nzval);
    return add_csc(c, c->flux_r, c->flux_c, c->flux_v, n, colptr, rowval, nzval);
}

static GainStage& gain_stage(dtb_ctx* c, int out, int in1, int in2) {
    auto key = std::make_tuple(out, in1, in2);
    auto it = c->gains.find(key);
    if (it == c->gains.end()) {
        GainStage g;
        g.out = out;
        g.in1 = in1;
        g.in2 = in2;
        it = c->gains.emplace(key, std::move(g)).first;
    }
    return it->second;
}

int32_t dtb_add_gain_block(dtb_ctx* c, int32_t out_sp, int32_t in1_sp, int32_t in2_sp, const void* G, int32_t dtype,
                           int32_t on_device) {
    DTB_CHECK(c && G, DTB_EINVAL, "dtb_add_gain_block: null argument");
    DTB_CHECK(!c->committed, DTB_ESTATE, "dtb_add_gain_block: operators already committed");
    DTB_CHECK(out_sp >= 0 && out_sp < c->ns && in1_sp >= 0 && in1_sp < c->ns && in2_sp >= 0 && in2_sp < c->ns,
              DTB_EINVAL, "dtb_add_gain_block: species index out of range");
    DTB_CHECK(dtype == DTB_DTYPE_F64 || dtype == DTB_DTYPE_F32, DTB_EINVAL, "dtb_add_gain_block: bad dtype");
    const int64_t no = c->sz[out_sp], n1 = c->sz[in1_sp], n2 = c->sz[in2_sp];
    if (on_device) {
        DTB_CHECK(in1_sp <= in2_sp, DTB_EINVAL, "dtb_add_gain_block: device blocks need in1_sp <= in2_sp");
        GainStage& g = gain_stage(c, out_sp, in1_sp, in2_sp);
        g.dev_src.emplace_back(G, dtype);
        return DTB_OK;
    }
    // host: FP64 accumulation, transposed to in1 <= in2
    const bool swap = in1_sp > in2_sp;
    GainStage& g = swap ? gain_stage(c, out_sp, in2_sp, in1_sp) : gain_stage(c, out_sp, in1_sp, in2_sp);
    if (g.host.empty()) g.host.assign((size_t)(no * n1 * n2), 0.0);
    for (int64_t a = 0; a < no; ++a)
        for (int64_t b = 0; b < n1; ++b)
            for (int64_t cc = 0; cc < n2; ++cc) {
                const size_t src = (size_t)((a * n1 + b) * n2 + cc);
                const double v = dtype == DTB_DTYPE_F64 ? static_cast<const double*>(G)[src]
                                                        : (double)static_cast<const float*>(G)[src];
                const size_t dst = swap ? (size_t)((a * n2 + cc) * n1 + b) : src;
                g.host[dst] += v;
            }
    return DTB_OK;
}

int32_t dtb_add_loss_block(dtb_ctx* c, int32_t sp, int32_t other_sp, const double* L) {
    DTB_CHECK(c && L, DTB_EINVAL, "dtb_add_loss_block: null argument");
    DTB_CHECK(!c->committed, DTB_ESTATE, "dtb_add_loss_block: operators already committed");
    DTB_CHECK(sp >= 0 && sp < c->ns && other_sp >= 0 && other_sp < c->ns, DTB_EINVAL,
              "dtb_add_loss_block: species index out of range");
    auto& v = c->losses[{sp, other_sp}];
    const size_t n = (size_t)(c->sz[sp] * c->sz[other_sp]);
    if (v.empty()) v.assign(n, 0.0);
    for (size_t i = 0; i < n; ++i) v[i] += L[i];
    return DTB_OK;
}

int32_t dtb_upload_mbin_csc(dtb_ctx* c, int64_t n_mom, const int64_t* colptr, const int64_t* rowval,
                            const double* nzval) {
    DTB_CHECK(c && colptr, DTB_EINVAL, "dtb_upload_mbin_csc: null argument");
    DTB_CHECK(!c->committed, DTB_ESTATE, "dtb_upload_mbin_csc: operators already committed");
    DTB_CHECK(n_mom == c->n_mom, DTB_EINVAL, "dtb_upload_mbin_csc: M_Bin must be n_mom^2 x n_mom (SteppingMethods.jl:349)");
    const int64_t N = n_mom, base = c->opts.index_base;
    DTB_CHECK(colptr[0] == base, DTB_EINVAL, "dtb_upload_mbin_csc: colptr[0] must equal index_base");
    DTB_CHECK(colptr[N] == colptr[0] || (rowval && nzval), DTB_EINVAL, "dtb_upload_mbin_csc: null rowval/nzval");
    for (int64_t k = 0; k < N; ++k) {
        DTB_CHECK(colptr[k + 1] >= colptr[k], DTB_EINVAL, "dtb_upload_mbin_csc: colptr not monotone");
        const int sk = species_of(c, k);
        for (int64_t p = colptr[k] - base; p < colptr[k + 1] - base; ++p) {
            const int64_t row = rowval[p] - base;
            DTB_CHECK(row >= 0 && row < N * N, DTB_EINVAL, "dtb_upload_mbin_csc: row index out of range");
            const double v = nzval[p];
            if (v == 0.0) continue;
            // M_Bin[(j - 1) N + a, k] is T[a, j, k]: df_a += T[a, j, k] f_j f_k
            const int64_t j = row / N, a = row - j * N;
            const int so = species_of(c, a), sj = species_of(c, j);
            const int64_t al = a - c->off[so];
            if (j == a || k == a) {
                // loss form: f_a * L'[a, c] f_c with c the other index (the row kernel subtracts)
                const int64_t o = j == a ? k : j;
                const int so2 = j == a ? sk : sj;
                auto& L = c->losses[{so, so2}];
                if (L.empty()) L.assign((size_t)(c->sz[so] * c->sz[so2]), 0.0);
                L[(size_t)(al * c->sz[so2] + (o - c->off[so2]))] -= v;
                continue;
            }
            // gain, folded to in1 <= in2 (G[a][b][c] = T[a,b,c] + T[a,c,b] across species)
            const bool swap = sj > sk;
            const int s1 = swap ? sk : sj, s2 = swap ? sj : sk;
            const int64_t b = swap ? k : j, cc = swap ? j : k;
            SparseGain& g = c->sgains[std::make_tuple(so, s1, s2)];
            g.a.push_back((int32_t)al);
            g.b.push_back((int32_t)(b - c->off[s1]));
            g.c.push_back((int32_t)(cc - c->off[s2]));
            g.v.push_back(v);
        }
    }
    return DTB_OK;
}

int32_t dtb_upload_mbin_ref(dtb_ctx* c, const double* M, int64_t n_mom) {
    DTB_CHECK(c && M, DTB_EINVAL, "dtb_upload_mbin_ref: null argument");
    DTB_CHECK(!c->committed, DTB_ESTATE, "dtb_upload_mbin_ref: operators already committed");
    DTB_CHECK(n_mom == c->n_mom, DTB_EINVAL, "dtb_upload_mbin_ref: M_Bin must be n_mom^2 x n_mom (SteppingMethods.jl:349)");
    const int64_t N = n_mom;
    const int64_t NN = N * N;
    // T[a,j,k] = M[(j*N + a) + k*N^2]. Exact split: loss-form rows collect the entries with j == a
    // or k == a (their contribution is f_a * sum_c L'[a,c] f_c); the rest is a gain tensor
    // folded to in1 <= in2.
    auto T = [&](int64_t a, int64_t j, int64_t k) { return M[(j * N + a) + k * NN]; };
    for (int so = 0; so < c->ns; ++so)
        for (int s1 = 0; s1 < c->ns; ++s1)
            for (int s2 = s1; s2 < c->ns; ++s2) {
                const int64_t no = c->sz[so], n1 = c->sz[s1], n2 = c->sz[s2];
                std::vector<double> blk((size_t)(no * n1 * n2), 0.0);
                bool nz = false;
                for (int64_t al = 0; al < no; ++al) {
                    const int64_t a = c->off[so] + al;
                    for (int64_t bl = 0; bl < n1; ++bl) {
                        const int64_t j = c->off[s1] + bl;
                        if (j == a) continue;
                        for (int64_t cl = 0; cl < n2; ++cl) {
                            const int64_t k = c->off[s2] + cl;
                            if (k == a) continue;
                            double v = T(a, j, k);
                            if (s1 != s2) v += T(a, k, j);
                            if (v != 0.0) nz = true;
                            blk[(size_t)((al * n1 + bl) * n2 + cl)] = v;
                        }
                    }
                }
                if (nz) {
                    GainStage& g = gain_stage(c, so, s1, s2);
                    if (g.host.empty()) g.host.assign(blk.size(), 0.0);
                    for (size_t i = 0; i < blk.size(); ++i) g.host[i] += blk[i];
                }
            }
    for (int sa = 0; sa < c->ns; ++sa)
        for (int sc = 0; sc < c->ns; ++sc) {
            const int64_t na = c->sz[sa], nc = c->sz[sc];
            std::vector<double> L((size_t)(na * nc), 0.0);
            bool nz = false;
            for (int64_t al = 0; al < na; ++al) {
                const int64_t a = c->off[sa] + al;
                for (int64_t cl = 0; cl < nc; ++cl) {
                    const int64_t k = c->off[sc] + cl;
                    double v = T(a, a, k);
                    if (k != a) v += T(a, k, a);
                    if (v != 0.0) nz = true;
                    L[(size_t)(al * nc + cl)] = -v;  // the kernel subtracts f_a * L f
                }
            }
            if (nz) {
                auto& v = c->losses[{sa, sc}];
                if (v.empty()) v.assign(L.size(), 0.0);
                for (size_t i = 0; i < L.size(); ++i) v[i] += L[i];
            }
        }
    return DTB_OK;
}

int32_t dtb_add_emi_block(dtb_ctx* c, int64_t row0, int64_t nrows, int64_t col0, int64_t ncols, const double* E) {
    DTB_CHECK(c && E, DTB_EINVAL, "dtb_add_emi_block: null argument");
    DTB_CHECK(!c->committed, DTB_ESTATE, "dtb_add_emi_block: operators already committed");
    DTB_CHECK(row0 >= 0 && nrows > 0 && row0 + nrows <= c->n_state && col0 >= 0 && ncols > 0 &&
                  col0 + ncols <= c->n_state,
              DTB_EINVAL, "dtb_add_emi_block: piece outside the n x n matrix");
    EmiPiece p{row0, nrows, col0, ncols, std::vector<double>(E, E + nrows * ncols)};
    c->emis.push_back(std::move(p));
    return DTB_OK;
}

int32_t dtb_upload_emi_ref(dtb_ctx* c, const double* M, int64_t n) {
    DTB_CHECK(c && M, DTB_EINVAL, "dtb_upload_emi_ref: null argument");
    DTB_CHECK(n == c->n_state, DTB_EINVAL, "dtb_upload_emi_ref: M_Emi must be n x n");
    // nonzero (cell, species) x (cell, species) pieces
    const int ng = c->n_space * c->ns;
    for (int gr = 0; gr < ng; ++gr)
        for (int gc = 0; gc < ng; ++gc) {
            const int64_t r0 = (gr / c->ns) * c->n_mom + c->off[gr % c->ns], nr = c->sz[gr % c->ns];
            const int64_t c0 = (gc / c->ns) * c->n_mom + c->off[gc % c->ns], nc = c->sz[gc % c->ns];
            std::vector<double> d((size_t)(nr * nc));
            bool nz = false;
            for (int64_t r = 0; r < nr; ++r)
                for (int64_t cc = 0; cc < nc; ++cc) {
                    const double v = M[(r0 + r) + (c0 + cc) * n];
                    d[(size_t)(r * nc + cc)] = v;
                    if (v != 0.0) nz = true;
                }
            if (nz) DTB_TRY(dtb_add_emi_block(c, r0, nr, c0, nc, d.data()));
        }
    return DTB_OK;
}

int32_t dtb_upload_vectors(dtb_ctx* c, const double* Ap, const double* Vol, const double* f_init, const double* inj) {
    DTB_CHECK(c && Ap && Vol && f_init && inj, DTB_EINVAL, "dtb_upload_vectors: null argument");
    DTB_CHECK(!c->committed, DTB_ESTATE, "dtb_upload_vectors: operators already committed");
    c->Ap.assign(Ap, Ap + c->n_state);
    c->Vol.assign(Vol, Vol + c->n_space);
    c->f_init.assign(f_init, f_init + c->n_state);
    c->inj.assign(inj, inj + c->n_state);
    c->have_vectors = true;
    return DTB_OK;
}

int32_t dtb_set_bin_domain(dtb_ctx* c, const int64_t* off_space, int64_t n) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_set_bin_domain: null context");
    DTB_CHECK(!c->committed, DTB_ESTATE, "dtb_set_bin_domain: operators already committed");
    if (!off_space || n < 0) {
        c->has_bin_domain = false;
        c->bin_domain.clear();
        return DTB_OK;
    }
    c->has_bin_domain = true;
    c->bin_domain.assign(off_space, off_space + n);
    return DTB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ commit
// CSR with duplicates summed, then a banded ELL of width w (max row length rounded to 4);
// padding slots have column -1.
template <typename T>
static int build_ell(dtb_ctx* c, const std::vector<int64_t>& fr, const std::vector<int64_t>& fc,
                     const std::vector<double>& fv, int& w_out, const T*& val_out, const int*& col_out) {
    const int64_t n = c->n_state;
    std::vector<std::vector<std::pair<int64_t, double>>> rows((size_t)n);
    for (size_t p = 0; p < fr.size(); ++p) rows[(size_t)fr[p]].push_back({fc[p], fv[p]});
    int w = 0;
    for (auto& r : rows) {
        std::stable_sort(r.begin(), r.end(), [](auto& x, auto& y) { return x.first < y.first; });
        std::vector<std::pair<int64_t, double>> m;
        for (auto& e : r) {
            if (!m.empty() && m.back().first == e.first)
                m.back().second += e.second;
            else
                m.push_back(e);
        }
        r.swap(m);
        w = std::max<int>(w, (int)r.size());
    }
    w = (int)round_up(std::max(w, 1), 4);
    std::vector<double> val((size_t)(n * w), 0.0);
    std::vector<int> col((size_t)(n * w), -1);
    for (int64_t i = 0; i < n; ++i)
        for (size_t k = 0; k < rows[(size_t)i].size(); ++k) {
            col[(size_t)i * w + k] = (int)rows[(size_t)i][k].first;
            val[(size_t)i * w + k] = rows[(size_t)i][k].second;
        }
    T* d_val;
    int* d_col;
    DTB_TRY(copy_host_vec(c, &d_val, val));
    DTB_TRY(copy_host_ints(c, &d_col, col));
    w_out = w;
    val_out = d_val;
    col_out = d_col;
    return DTB_OK;
}

// Sparse gain block layout: per output row, runs of consecutive nonzero b-rows, each run
// trimmed to the union of its rows' c-spans (8-element aligned). A run is cut where the union
// would pad the stored rows by more than half, where b skips a row, or at max_elems.
struct SparseRun {
    int al, b0, nb, c0, w;  // output row, first b, b-rows, first c, row width (elements)
    int64_t elem_off;       // within the sparse data
};

static void sparse_runs(const SparseGain& g, int64_t n2p, int64_t max_elems, std::vector<SparseRun>& runs,
                        std::vector<double>& data) {
    std::vector<size_t> idx(g.v.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) {
        if (g.a[x] != g.a[y]) return g.a[x] < g.a[y];
        if (g.b[x] != g.b[y]) return g.b[x] < g.b[y];
        return g.c[x] < g.c[y];
    });
    // rows (a, b) with their c-span
    struct Row {
        int a, b, c0, c1;
        size_t i0, i1;
    };
    std::vector<Row> rows;
    for (size_t k = 0; k < idx.size();) {
        size_t e = k;
        const int a = g.a[idx[k]], b = g.b[idx[k]];
        while (e < idx.size() && g.a[idx[e]] == a && g.b[idx[e]] == b) ++e;
        const int c0 = g.c[idx[k]] / 8 * 8;
        const int c1 = (int)std::min<int64_t>(n2p, round_up(g.c[idx[e - 1]] + 1, 8));
        rows.push_back({a, b, c0, c1, k, e});
        k = e;
    }
    auto flush = [&](size_t r0, size_t r1, int c0, int c1) {
        SparseRun R;
        R.al = rows[r0].a;
        R.b0 = rows[r0].b;
        R.nb = (int)(r1 - r0);
        R.c0 = c0;
        R.w = c1 - c0;
        R.elem_off = (int64_t)data.size();
        data.resize(data.size() + (size_t)R.nb * R.w, 0.0);
        for (size_t r = r0; r < r1; ++r)
            for (size_t q = rows[r].i0; q < rows[r].i1; ++q)
                data[(size_t)(R.elem_off + (int64_t)(r - r0) * R.w + (g.c[idx[q]] - c0))] += g.v[idx[q]];
        runs.push_back(R);
    };
    size_t r0 = 0;
    int u0 = 0, u1 = 0;
    int64_t own = 0;  // sum of the run's own row widths
    for (size_t r = 0; r < rows.size(); ++r) {
        if (r > r0) {
            const bool adj = rows[r].a == rows[r - 1].a && rows[r].b == rows[r - 1].b + 1;
            const int n0 = std::min(u0, rows[r].c0), n1 = std::max(u1, rows[r].c1);
            const int64_t padded = (int64_t)(r - r0 + 1) * (n1 - n0);
            const int64_t own2 = own + (rows[r].c1 - rows[r].c0);
            if (adj && 2 * padded <= 3 * own2 && padded <= max_elems) {
                u0 = n0;
                u1 = n1;
                own = own2;
                continue;
            }
            flush(r0, r, u0, u1);
        }
        r0 = r;
        u0 = rows[r].c0;
        u1 = rows[r].c1;
        own = u1 - u0;
    }
    if (!rows.empty()) flush(r0, rows.size(), u0, u1);
}

template <typename T>
static int commit_typed(dtb_ctx* c, RowOps<T>& ops) {
    const size_t esz = sizeof(T);
    // sparse entries of a block that also has dense host uploads are folded into the dense block
    for (auto it = c->sgains.begin(); it != c->sgains.end();) {
        auto dn = c->gains.find(it->first);
        if (dn == c->gains.end()) {
            ++it;
            continue;
        }
        GainStage& g = dn->second;
        DTB_CHECK(g.dev_src.empty(), DTB_EINVAL, "a sparse M_Bin cannot be summed with a device-resident gain block");
        const int64_t n1 = c->sz[g.in1], n2 = c->sz[g.in2];
        if (g.host.empty()) g.host.assign((size_t)(c->sz[g.out] * n1 * n2), 0.0);
        const SparseGain& s = it->second;
        for (size_t q = 0; q < s.v.size(); ++q) g.host[(size_t)(((int64_t)s.a[q] * n1 + s.b[q]) * n2 + s.c[q])] += s.v[q];
        it = c->sgains.erase(it);
    }
    // ---------------- gain blocks
    struct BlkInfo {
        int out, in1, in2;
        int64_t no, n1, n2, n2p;
        int64_t elem_off;
    };
    std::vector<BlkInfo> blks;
    int64_t total_elems = 0;
    for (auto& kv : c->gains) {
        GainStage& g = kv.second;
        BlkInfo b{g.out, g.in1, g.in2, c->sz[g.out], c->sz[g.in1], c->sz[g.in2], round_up(c->sz[g.in2], 8), 0};
        DTB_CHECK(b.n2p * (int64_t)esz <= kGainTileBytes, DTB_EINVAL,
                  "gain block input-2 species has too many states for one staged b-row");
        total_elems = round_up(total_elems, 256 / (int64_t)esz);
        b.elem_off = total_elems;
        total_elems += b.no * b.n1 * b.n2p;
        blks.push_back(b);
    }
    // sparse blocks: runs built on the host, their data placed after the dense blocks
    struct SpBlk {
        int out, in1, in2;
        std::vector<SparseRun> runs;
        int64_t elem_off;
    };
    std::vector<SpBlk> sblks;
    std::vector<double> sdata;
    double sparse_bytes = 0;
    for (auto& kv : c->sgains) {
        SpBlk sb;
        sb.out = std::get<0>(kv.first);
        sb.in1 = std::get<1>(kv.first);
        sb.in2 = std::get<2>(kv.first);
        const int64_t n2p = round_up(c->sz[sb.in2], 8);
        DTB_CHECK(n2p * (int64_t)esz <= kGainTileBytes, DTB_EINVAL,
                  "gain block input-2 species has too many states for one staged b-row");
        sdata.clear();
        sparse_runs(kv.second, n2p, (int64_t)(64 * 1024 / esz), sb.runs, sdata);
        total_elems = round_up(total_elems, 256 / (int64_t)esz);
        sb.elem_off = total_elems;
        total_elems += (int64_t)sdata.size();
        sparse_bytes += (double)sdata.size() * esz;
        // staged now: the host copy of this block's data goes with it
        std::vector<T> tv(sdata.size());
        for (size_t i = 0; i < sdata.size(); ++i) tv[i] = (T)sdata[i];
        sb.runs.shrink_to_fit();
        sblks.push_back(std::move(sb));
        c->sparse_stage.emplace_back(reinterpret_cast<const char*>(tv.data()),
                                     reinterpret_cast<const char*>(tv.data()) + tv.size() * esz);
    }
    c->has_bin = !c->gains.empty() || !c->losses.empty() || !c->sgains.empty();
    if (!blks.empty() || !sblks.empty()) {
        DTB_TRY(c->alloc(&c->G_all, esz * (size_t)total_elems));
        DTB_CUDA(cudaMemsetAsync(c->G_all, 0, esz * (size_t)total_elems, c->stream));
        for (size_t k = 0; k < sblks.size(); ++k) {
            const auto& st = c->sparse_stage[k];
            if (!st.empty())
                DTB_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(c->G_all) + esz * (size_t)sblks[k].elem_off, st.data(),
                                         st.size(), cudaMemcpyHostToDevice, c->stream));
        }
        DTB_CUDA(cudaStreamSynchronize(c->stream));
        c->sparse_stage.clear();
        c->sgains.clear();
        size_t bi = 0;
        for (auto& kv : c->gains) {
            GainStage& g = kv.second;
            const BlkInfo& b = blks[bi++];
            T* dst = reinterpret_cast<T*>(c->G_all) + b.elem_off;
            const int64_t rows = b.no * b.n1;
            if (!g.host.empty()) {
                // host FP64 -> T, padded rows, through chunks
                const int64_t chunk_rows = std::max<int64_t>(1, (64ll << 20) / (b.n2p * (int64_t)esz));
                std::vector<T> tmp;
                for (int64_t r0 = 0; r0 < rows; r0 += chunk_rows) {
                    const int64_t nr = std::min(chunk_rows, rows - r0);
                    tmp.assign((size_t)(nr * b.n2p), T(0));
                    for (int64_t r = 0; r < nr; ++r)
                        for (int64_t k = 0; k < b.n2; ++k)
                            tmp[(size_t)(r * b.n2p + k)] = (T)g.host[(size_t)((r0 + r) * b.n2 + k)];
                    DTB_CUDA(cudaMemcpyAsync(dst + r0 * b.n2p, tmp.data(), sizeof(T) * tmp.size(),
                                             cudaMemcpyHostToDevice, c->stream));
                    DTB_CUDA(cudaStreamSynchronize(c->stream));
                }
            }
            for (auto& src : g.dev_src) {
                DTB_CHECK(g.host.empty() && g.dev_src.size() == 1, DTB_EINVAL,
                          "a device-resident gain block cannot be summed with other uploads of the same block");
                cudaError_t e;
                if (src.second == DTB_DTYPE_F64)
                    e = launch_pad_rows<double, T>(static_cast<const double*>(src.first), rows, (int)b.n2, dst,
                                                   (int)b.n2p, c->stream);
                else
                    e = launch_pad_rows<float, T>(static_cast<const float*>(src.first), rows, (int)b.n2, dst,
                                                  (int)b.n2p, c->stream);
                DTB_CUDA(e);
                DTB_CUDA(cudaStreamSynchronize(c->stream));
            }
            g.host.clear();
            g.host.shrink_to_fit();
        }
    }
    // work units, ordered by output row
    c->f_smem_len = (int)c->offp[c->ns];
    int bps = gain_stream_blocks_per_sm((int)esz, c->f_smem_len);
    DTB_CHECK(bps >= 1 || (blks.empty() && sblks.empty()), DTB_EINVAL,
              "gain kernel does not fit on an SM (state vector too long)");
    if (bps < 1) bps = 1;
    std::vector<GainUnit> units;
    std::vector<int> unit_ptr((size_t)c->n_mom + 1, 0);
    {
        double tot_bytes = sparse_bytes;
        for (auto& b : blks) tot_bytes += (double)b.no * b.n1 * b.n2 * esz;
        c->gain_bytes = tot_bytes;
        // sparse runs per output row (global momentum index)
        std::vector<std::vector<std::pair<const SpBlk*, const SparseRun*>>> srow((size_t)c->n_mom);
        for (auto& sb : sblks)
            for (auto& R : sb.runs) srow[(size_t)(c->off[sb.out] + R.al)].push_back({&sb, &R});
        // about 8 work units per CTA spread the HBM stream of a large G evenly; an L2-resident G
        // (64 MB or less) is bound by the per-unit round trip of the tile ring instead, so its
        // units are about 8 times larger (config 0: 14.8 against 15.6 us per step)
        const double units_per_cta = tot_bytes <= 64.0 * 1024 * 1024 ? 1.0 : 8.0;
        const double target = std::min(256.0 * 1024, std::max((double)kGainTileBytes,
                                                               tot_bytes / ((double)c->num_sms * bps * units_per_cta)));
        for (int64_t a = 0; a < c->n_mom; ++a) {
            unit_ptr[(size_t)a] = (int)units.size();
            const int sa = species_of(c, a);
            for (auto& b : blks) {
                if (b.out != sa) continue;
                const int64_t al = a - c->off[sa];
                const int64_t row_b = b.n2p * (int64_t)esz;
                const int tile_b = (int)std::max<int64_t>(1, std::min<int64_t>(b.n1, kGainTileBytes / row_b));
                int64_t nb = std::max<int64_t>(tile_b, (int64_t)(target / row_b) / tile_b * tile_b);
                for (int64_t b0 = 0; b0 < b.n1; b0 += nb) {
                    GainUnit u;
                    u.g_off = b.elem_off + (al * b.n1 + b0) * b.n2p;
                    u.b_off = (int)(c->offp[b.in1] + b0);
                    u.c_off = (int)c->offp[b.in2];
                    u.nb = (int)std::min(nb, b.n1 - b0);
                    u.n2p = (int)b.n2p;
                    u.tile_b = tile_b;
                    u.row = (int)a;
                    units.push_back(u);
                }
            }
            for (auto& pr : srow[(size_t)a]) {
                const SpBlk& sb = *pr.first;
                const SparseRun& R = *pr.second;
                const int tile_b = (int)std::max<int64_t>(1, std::min<int64_t>(R.nb, kGainTileBytes / (R.w * (int64_t)esz)));
                GainUnit u;
                u.g_off = sb.elem_off + R.elem_off;
                u.b_off = (int)(c->offp[sb.in1] + R.b0);
                u.c_off = (int)(c->offp[sb.in2] + R.c0);
                u.nb = R.nb;
                u.n2p = R.w;
                u.tile_b = tile_b;
                u.row = (int)a;
                units.push_back(u);
            }
        }
        unit_ptr[(size_t)c->n_mom] = (int)units.size();
    }
    c->n_units = (int)units.size();
    c->gain_grid = std::max(1, std::min(c->n_units, c->num_sms * bps));
    DTB_TRY(copy_host_ints(c, &c->units, units));
    DTB_TRY(copy_host_ints(c, &c->unit_ptr, unit_ptr));
    DTB_TRY(c->alloc(&c->partial, sizeof(double) * (size_t)std::max(1, c->n_units) * c->n_space));
    DTB_CUDA(cudaMemsetAsync(c->partial, 0, sizeof(double) * (size_t)std::max(1, c->n_units) * c->n_space,
                             c->stream));

    // ---------------- loss blocks, grouped by row species
    {
        std::vector<long long> doff;
        std::vector<int> ld, coff, ncols;
        std::vector<double> data;
        for (int s = 0; s < c->ns; ++s) {
            ops.loss_ptr[s] = (int)doff.size();
            for (auto& kv : c->losses) {
                if (kv.first.first != s) continue;
                const int oth = kv.first.second;
                const int64_t nr = c->sz[s], nc = c->sz[oth], l = round_up(nc, 4);
                doff.push_back((long long)data.size());
                ld.push_back((int)l);
                coff.push_back((int)c->off[oth]);
                ncols.push_back((int)nc);
                const size_t base = data.size();
                data.resize(base + (size_t)(nr * l), 0.0);
                for (int64_t r = 0; r < nr; ++r)
                    for (int64_t k = 0; k < nc; ++k) data[base + (size_t)(r * l + k)] = kv.second[(size_t)(r * nc + k)];
            }
        }
        ops.loss_ptr[c->ns] = (int)doff.size();
        long long* d_doff;
        int *d_ld, *d_coff, *d_nc;
        T* d_data;
        DTB_TRY(copy_host_ints(c, &d_doff, doff));
        DTB_TRY(copy_host_ints(c, &d_ld, ld));
        DTB_TRY(copy_host_ints(c, &d_coff, coff));
        DTB_TRY(copy_host_ints(c, &d_nc, ncols));
        DTB_TRY(copy_host_vec(c, &d_data, data));
        ops.loss_data_off = d_doff;
        ops.loss_ld = d_ld;
        ops.loss_col_off = d_coff;
        ops.loss_ncols = d_nc;
        ops.loss_data = d_data;
    }
    // ---------------- emission pieces, per row lists
    {
        c->has_emi = !c->emis.empty();
        std::vector<long long> doff;
        std::vector<int> ld, r0v, c0v, ncv;
        std::vector<double> data;
        std::vector<std::vector<int>> rows((size_t)c->n_state);
        for (size_t p = 0; p < c->emis.size(); ++p) {
            const EmiPiece& e = c->emis[p];
            const int64_t l = round_up(e.ncols, 4);
            doff.push_back((long long)data.size());
            ld.push_back((int)l);
            r0v.push_back((int)e.row0);
            c0v.push_back((int)e.col0);
            ncv.push_back((int)e.ncols);
            const size_t base = data.size();
            data.resize(base + (size_t)(e.nrows * l), 0.0);
            for (int64_t r = 0; r < e.nrows; ++r) {
                for (int64_t k = 0; k < e.ncols; ++k) data[base + (size_t)(r * l + k)] = e.data[(size_t)(r * e.ncols + k)];
                rows[(size_t)(e.row0 + r)].push_back((int)p);
            }
        }
        std::vector<int> rptr((size_t)c->n_state + 1, 0), piece;
        for (int64_t i = 0; i < c->n_state; ++i) {
            rptr[(size_t)i] = (int)piece.size();
            for (int p : rows[(size_t)i]) piece.push_back(p);
        }
        rptr[(size_t)c->n_state] = (int)piece.size();
        int *d_rptr, *d_piece, *d_ld, *d_r0, *d_c0, *d_nc;
        long long* d_doff;
        T* d_data;
        DTB_TRY(copy_host_ints(c, &d_rptr, rptr));
        DTB_TRY(copy_host_ints(c, &d_piece, piece));
        DTB_TRY(copy_host_ints(c, &d_doff, doff));
        DTB_TRY(copy_host_ints(c, &d_ld, ld));
        DTB_TRY(copy_host_ints(c, &d_r0, r0v));
        DTB_TRY(copy_host_ints(c, &d_c0, c0v));
        DTB_TRY(copy_host_ints(c, &d_nc, ncv));
        DTB_TRY(copy_host_vec(c, &d_data, data));
        ops.emi_rptr = d_rptr;
        ops.emi_piece = d_piece;
        ops.emi_data_off = d_doff;
        ops.emi_ld = d_ld;
        ops.emi_row0 = d_r0;
        ops.emi_col0 = d_c0;
        ops.emi_ncols = d_nc;
        ops.emi_data = d_data;
    }
    // ---------------- flux: CSR with duplicates summed, then banded ELL (X + P, or P and X
    // separately for the symplectic method)
    DTB_TRY(build_ell<T>(c, c->flux_r, c->flux_c, c->flux_v, ops.ell_w, ops.ell_val, ops.ell_col));
    if (c->symplectic) {
        DTB_TRY(build_ell<T>(c, c->xflux_r, c->xflux_c, c->xflux_v, ops.x_ell_w, ops.x_ell_val, ops.x_ell_col));
        T *fm, *dfm;
        DTB_TRY(c->alloc(&fm, sizeof(T) * (size_t)c->n_state));
        DTB_TRY(c->alloc(&dfm, sizeof(T) * (size_t)c->n_state));
        c->fm_buf = fm;
        c->dfm_buf = dfm;
        ops.dfm_out = dfm;
    }
    ops.mode = 0;
    ops.thr_mom = c->prec == DTB_F64 ? (double)1e-10f : (double)(T)1e-10f;
    ops.thr_space = c->prec == DTB_F64 ? (double)1e-20f : (double)(T)1e-20f;
    // ---------------- vectors
    {
        std::vector<double> invAp(c->Ap.size());
        for (size_t i = 0; i < invAp.size(); ++i) invAp[i] = (double)((T)1 / (T)c->Ap[i]);  // SteppingStructs.jl:55
        T *d_inv, *d_inj, *d_vol;
        DTB_TRY(copy_host_vec(c, &d_inv, invAp));
        DTB_TRY(copy_host_vec(c, &d_inj, c->inj));
        DTB_TRY(copy_host_vec(c, &d_vol, c->Vol));
        ops.invAp = d_inv;
        ops.inj = d_inj;
        ops.vol = d_vol;
        T* fi;
        DTB_TRY(copy_host_vec(c, &fi, c->f_init));
        c->f_init_dev = fi;
        DTB_TRY(c->alloc(reinterpret_cast<T**>(&c->f_buf[0]), sizeof(T) * (size_t)c->n_state));
        DTB_TRY(c->alloc(reinterpret_cast<T**>(&c->f_buf[1]), sizeof(T) * (size_t)c->n_state));
        DTB_CUDA(cudaMemcpyAsync(c->f_buf[0], fi, sizeof(T) * (size_t)c->n_state, cudaMemcpyDeviceToDevice,
                                 c->stream));
        c->cur = 0;
    }
    ops.n_mom = (int)c->n_mom;
    ops.n_state = (int)c->n_state;
    ops.n_space = c->n_space;
    ops.n_species = c->ns;
    for (int s = 0; s <= c->ns; ++s) {
        ops.sp_off[s] = (int)c->off[s];
        ops.sp_offp[s] = (int)c->offp[s];
        c->sp_off_host[s] = (int)c->off[s];
        c->sp_off_host[c->ns + 1 + s] = (int)c->offp[s];
    }
    ops.unit_ptr = c->unit_ptr;
    ops.n_units = c->n_units;
    ops.partial = c->partial;
    ops.thr = c->prec == DTB_F64 ? (double)1e-10f : (double)(T)1e-10f;
    // binary domain: `in(off_space, Domain)` per cell (entries outside 0..n_space-1 match no cell)
    ops.bin_on = nullptr;
    c->n_bin_cells = c->n_space;
    c->bin_cells = nullptr;
    if (c->has_bin_domain) {
        std::vector<int> on((size_t)c->n_space, 0), list;
        for (int64_t k : c->bin_domain)
            if (k >= 0 && k < c->n_space) on[(size_t)k] = 1;
        for (int k = 0; k < c->n_space; ++k)
            if (on[(size_t)k]) list.push_back(k);
        std::vector<unsigned char> on8(on.begin(), on.end());
        unsigned char* d_on;
        DTB_TRY(c->alloc(&d_on, on8.size()));
        DTB_CUDA(cudaMemcpyAsync(d_on, on8.data(), on8.size(), cudaMemcpyHostToDevice, c->stream));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
        ops.bin_on = d_on;
        c->n_bin_cells = (int)list.size();
        if (!list.empty()) DTB_TRY(copy_host_ints(c, &c->bin_cells, list));
    }
    ops.has_bin = c->has_bin;
    ops.has_emi = c->has_emi;
    return DTB_OK;
}

extern "C" int32_t dtb_commit(dtb_ctx* c) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_commit: null context");
    if (c->committed) return DTB_OK;
    DTB_RANGE("dtb_commit");
    DTB_CHECK(c->have_vectors, DTB_ESTATE, "dtb_commit: dtb_upload_vectors was not called");
    DeviceGuard g(c->device);
    if (c->prec == DTB_MIXED) {
        int rc = commit_mixed(c);
        if (rc != DTB_OK) {
            destroy_mixed(c);
            c->free_all();
            return rc;
        }
        c->committed = true;
        c->gains.clear();
        c->losses.clear();
        c->emis.clear();
        c->flux_r.clear();
        c->flux_c.clear();
        c->flux_v.clear();
        return DTB_OK;
    }
    int rc = c->prec == DTB_F64 ? commit_typed<double>(c, c->ops_d) : commit_typed<float>(c, c->ops_f);
    if (rc != DTB_OK) {
        c->free_all();
        return rc;
    }
    DTB_TRY(c->alloc(&c->dt_arr, sizeof(double) * (size_t)c->hist_cap));
    DTB_TRY(c->alloc(&c->ctr, sizeof(unsigned long long)));
    DTB_TRY(c->alloc(&c->hist, sizeof(StepDiagDev) * (size_t)c->hist_cap));
    c->rows_grid = euler_rows_blocks((int)c->n_state);
    DTB_TRY(c->alloc(&c->blk_red, sizeof(double) * kStepRecFields * (size_t)c->rows_grid * c->graph_steps));
    DTB_TRY(c->alloc(&c->ticket, sizeof(unsigned)));
    DTB_TRY(c->alloc(&c->err, sizeof(int)));
    std::vector<int> spo(c->off, c->off + c->ns + 1);
    DTB_TRY(copy_host_ints(c, &c->sp_off_dev, spo));
    DTB_TRY(c->alloc(&c->mom_w, sizeof(double) * (size_t)c->n_mom));
    DTB_TRY(c->alloc(&c->mom_out, sizeof(double) * 2 * (size_t)c->ns * c->n_space));
    DTB_CUDA(cudaMemsetAsync(c->ctr, 0, sizeof(unsigned long long), c->stream));
    DTB_CUDA(cudaMemsetAsync(c->ticket, 0, sizeof(unsigned), c->stream));
    DTB_CUDA(cudaMemsetAsync(c->err, 0, sizeof(int), c->stream));
    DTB_CUDA(cudaMallocHost(&c->pin_dt, sizeof(double) * (size_t)c->hist_cap));
    DTB_CUDA(cudaMallocHost(&c->pin_hist, sizeof(StepDiagDev) * (size_t)c->hist_cap));
    DTB_CUDA(cudaMallocHost(&c->pin_err, sizeof(int)));
    if (c->prec == DTB_F32) DTB_CUDA(cudaMallocHost(&c->pin_f32, sizeof(float) * (size_t)c->n_state));
    DTB_CUDA(cudaDeviceSynchronize());
    c->host_ctr = 0;
    c->committed = true;
    // staging no longer needed
    c->gains.clear();
    c->losses.clear();
    c->emis.clear();
    c->flux_r.clear();
    c->flux_c.clear();
    c->flux_v.clear();
    return DTB_OK;
}

// ------------------------------------------------------------------ stepping internals
static int flush_profile(dtb_ctx* c) {
    if (c->prof_pending == 0) return DTB_OK;
    DTB_CUDA(cudaEventSynchronize(c->ev[(size_t)(2 * (c->prof_pending - 1) + 1)]));
    for (int k = 0; k < c->prof_pending; ++k) {
        float ms = 0;
        DTB_CUDA(cudaEventElapsedTime(&ms, c->ev[(size_t)(2 * k)], c->ev[(size_t)(2 * k + 1)]));
        c->prof_ms += ms;
    }
    c->prof_pending = 0;
    return DTB_OK;
}

// One step: number *ctr + kpos of the dt sequence, whose row blocks write record slot kpos;
// finish_seq reduces a sequence's records and advances the counter.
template <typename T>
static int launch_step(dtb_ctx* c, RowOps<T>& ops, double dt_imm, bool use_arr, int verbose, bool profile,
                       int kpos) {
    T* fin = reinterpret_cast<T*>(c->f_buf[c->cur]);
    T* fout = reinterpret_cast<T*>(c->f_buf[c->cur ^ 1]);
    const bool gain = c->n_units > 0 && c->n_bin_cells > 0;
    if (gain) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (profile) {
            const size_t k = (size_t)c->prof_pending * 2;
            while (c->ev.size() < k + 2) {
                cudaEvent_t e;
                DTB_CUDA(cudaEventCreate(&e));
                c->ev.push_back(e);
            }
            e0 = c->ev[k];
            e1 = c->ev[k + 1];
            DTB_CUDA(cudaEventRecord(e0, c->stream));
        }
        DTB_CUDA(launch_gain_stream<T>(reinterpret_cast<const T*>(c->G_all), c->units, c->n_units, fin, (int)c->n_mom,
                                       c->sp_off_host, c->ns, c->f_smem_len, c->partial, c->n_bin_cells,
                                       c->gain_grid, c->err, c->stream, c->bin_cells, true));
        c->launches++;
        if (profile) {
            DTB_CUDA(cudaEventRecord(e1, c->stream));
            c->prof_n++;
            if (++c->prof_pending == kProfRing) DTB_TRY(flush_profile(c));
        }
    }
    const double* dta = use_arr ? c->dt_arr : nullptr;
    double* rec = c->blk_red + (size_t)kpos * c->rows_grid * kStepRecFields;
    if (c->symplectic) {
        RowOps<T> mom = ops;
        mom.mode = 1;
        T* fm = reinterpret_cast<T*>(c->fm_buf);
        T* dfm = reinterpret_cast<T*>(c->dfm_buf);
        DTB_CUDA(launch_euler_rows<T>(mom, fin, fm, dt_imm, dta, c->ctr, kpos, verbose, nullptr, gain, c->stream));
        DTB_CUDA(launch_sympl_space<T>(ops, fin, fm, dfm, fout, dt_imm, dta, c->ctr, kpos, rec, c->stream));
        c->launches += 2;
    } else {
        DTB_CUDA(launch_euler_rows<T>(ops, fin, fout, dt_imm, dta, c->ctr, kpos, verbose, rec, gain, c->stream));
        c->launches++;
    }
    c->cur ^= 1;
    c->host_ctr++;
    return DTB_OK;
}

static int do_step(dtb_ctx* c, double dt_imm, bool use_arr, int verbose, bool profile, int kpos) {
    return c->prec == DTB_F64 ? launch_step<double>(c, c->ops_d, dt_imm, use_arr, verbose, profile, kpos)
                              : launch_step<float>(c, c->ops_f, dt_imm, use_arr, verbose, profile, kpos);
}

// The diagnostics of the last n steps (a sequence of record slots 0..n-1) and the counter advance.
static int finish_seq(dtb_ctx* c, int n, int verbose) {
    if (n <= 0) return DTB_OK;
    const int hb = c->prec == DTB_F64 ? c->ops_d.has_bin : c->ops_f.has_bin;
    const int he = c->prec == DTB_F64 ? c->ops_d.has_emi : c->ops_f.has_emi;
    DTB_CUDA(launch_step_diag(c->blk_red, c->rows_grid, n, c->ctr, c->hist, c->hist_cap, verbose, hb, he,
                              c->symplectic ? 1 : 0, c->ticket, c->stream));
    c->launches++;
    return DTB_OK;
}

// n steps outside a graph, in sequences of at most graph_steps (the record slots).
static int run_loose(dtb_ctx* c, int64_t n, int verbose, bool profile) {
    for (int64_t done = 0; done < n;) {
        const int m = (int)std::min<int64_t>(c->graph_steps, n - done);
        for (int k = 0; k < m; ++k) DTB_TRY(do_step(c, 0.0, true, verbose, profile, k));
        DTB_TRY(finish_seq(c, m, verbose));
        done += m;
    }
    return DTB_OK;
}

static int check_kernel_err(dtb_ctx* c) {
    DTB_CUDA(cudaMemcpyAsync(c->pin_err, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    if (*c->pin_err) {
        const int e = *c->pin_err;
        cudaMemsetAsync(c->err, 0, sizeof(int), c->stream);
        cudaStreamSynchronize(c->stream);
        set_error("a bounded device wait gave up (kernel error flags " + std::to_string(e) + ")");
        return DTB_ETIMEOUT;
    }
    return DTB_OK;
}

int batch_prepare(dtb_ctx* c);  // batch_api.cpp

static int ensure_graph(dtb_ctx* c, int verbose) {
    if (c->graph && c->graph_verbose == verbose) return DTB_OK;
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    const int saved_cur = c->cur;
    const unsigned long long saved_ctr = c->host_ctr;
    const long long saved_launches = c->launches;
    c->cur = 0;
    cudaGraph_t g;
    DTB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = DTB_OK;
    for (int k = 0; k < c->graph_steps && rc == DTB_OK; ++k) rc = do_step(c, 0.0, true, verbose, false, k);
    if (rc == DTB_OK) rc = finish_seq(c, c->graph_steps, verbose);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->graph_launches = c->launches - saved_launches;
    c->cur = saved_cur;
    c->host_ctr = saved_ctr;
    c->launches = saved_launches;
    if (rc != DTB_OK) return rc;
    DTB_CUDA(e);
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    DTB_CUDA(e);
    c->graph_verbose = verbose;
    return DTB_OK;
}

// Runs n steps whose dt/dt0 values are in pinned c->pin_dt[0..n) (n <= hist_cap); steps
// read them through the device counter, which is reset to 0 first.
static int run_chunk(dtb_ctx* c, int64_t n, int verbose, bool use_graph) {
    DTB_CUDA(cudaMemcpyAsync(c->dt_arr, c->pin_dt, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    DTB_CUDA(cudaMemsetAsync(c->ctr, 0, sizeof(unsigned long long), c->stream));
    c->host_ctr = 0;
    int64_t done = 0;
    if (use_graph && !c->profiling && n >= c->graph_steps) {
        if (c->cur != 0) {
            DTB_TRY(run_loose(c, 1, verbose, false));
            done++;
        }
        DTB_TRY(ensure_graph(c, verbose));
        while (n - done >= c->graph_steps) {
            DTB_CUDA(cudaGraphLaunch(c->graph, c->stream));
            done += c->graph_steps;
            c->host_ctr += c->graph_steps;
            c->launches += c->graph_launches;
        }
    }
    return run_loose(c, n - done, verbose, c->profiling);
}

static void print_cr(int verbose, const StepDiagDev& d, double t, double t_stop, double dt) {
    if (verbose == 1 && d.cr[0] > 1.0)
        std::printf("Cr = %.17g, t=%.17g, dt=%.17g, system may be unstable\n", d.cr[0], t, dt);
    else if (verbose == 2)
        std::printf("\rCr = %.17g, t=%.17g, dt=%.17g\n", d.cr[0], t, dt);
    else if (verbose == 3)
        std::printf("Cr = %.17g,Cr_Bin = %.17g, Cr_Emi = %.17g, Cr_Flux = %.17g, t=%.17g, t_save =%.17g, dt=%.17g\n",
                    d.cr[0], d.cr[1], d.cr[2], d.cr[3], t, t_stop, dt);
    if (!d.finite) std::printf("non-finite value in df calculation\n");
}

static double dt0_eff(const dtb_ctx* c) {
    return c->prec == DTB_F32 ? (double)(float)c->opts.dt0 : c->opts.dt0;
}

// The step of dtb_step, enqueued: dt truncated at t_stop (SteppingMethods.jl:18-27), the step's
// kernels and its diagnostics reduction; *idx gets the step's slot in the step history.
static int enqueue_step(dtb_ctx* c, double t_start, double t_stop, double* dt, int* save, int verbose,
                        unsigned long long* idx) {
    *save = 0;
    if (t_start + *dt >= t_stop) {
        *dt = t_stop - t_start;
        *save = 1;
    }
    const double dt_scale = *dt / dt0_eff(c);
    if (c->host_ctr >= (unsigned long long)c->hist_cap) {
        DTB_CUDA(cudaMemsetAsync(c->ctr, 0, sizeof(unsigned long long), c->stream));
        c->host_ctr = 0;
    }
    *idx = c->host_ctr;
    DTB_TRY(do_step(c, dt_scale, false, verbose, false, 0));
    DTB_TRY(finish_seq(c, 1, verbose));
    c->steps_run++;
    return DTB_OK;
}

extern "C" {

int32_t dtb_step(dtb_ctx* c, double t_start, double t_stop, double dt, int32_t verbose, double* dt_out,
                 int32_t* save_out, dtb_step_diag* diag_out) {
    DTB_RANGE("dtb_step");
    DTB_CHECK(c, DTB_EINVAL, "dtb_step: null context");
    DTB_CHECK(c->prec != DTB_MIXED, DTB_ESTATE, "dtb_step: batched contexts use the dtb_batch_* entry points");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    int save = 0;
    unsigned long long idx = 0;
    DTB_TRY(enqueue_step(c, t_start, t_stop, &dt, &save, verbose, &idx));
    if (dt_out) *dt_out = dt;
    if (save_out) *save_out = save;
    if (verbose == 1 || verbose == 2 || verbose == 3 || diag_out) {
        DTB_CUDA(cudaMemcpyAsync(c->pin_hist, c->hist + idx, sizeof(StepDiagDev), cudaMemcpyDeviceToHost, c->stream));
        DTB_TRY(check_kernel_err(c));
        if (diag_out) std::memcpy(diag_out, c->pin_hist, sizeof(StepDiagDev));
    }
    return DTB_OK;
}

int32_t dtb_step_io(dtb_ctx* c, const double* f_in, double* f_out, double t_start, double t_stop, double dt,
                    int32_t verbose, double* dt_out, int32_t* save_out, dtb_step_diag* diag_out) {
    DTB_RANGE("dtb_step_io");
    DTB_CHECK(c && f_out, DTB_EINVAL, "dtb_step_io: null argument");
    DTB_CHECK(c->prec != DTB_MIXED, DTB_ESTATE, "dtb_step_io: batched contexts use dtb_batch_run_io");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    const size_t n = (size_t)c->n_state;
    // the FP32 staging buffer is idle here: every call that fills or drains it waits for its copy
    if (f_in) {
        if (c->prec == DTB_F64) {
            DTB_CUDA(cudaMemcpyAsync(c->f_buf[c->cur], f_in, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
        } else {
            for (size_t k = 0; k < n; ++k) c->pin_f32[k] = (float)f_in[k];
            DTB_CUDA(cudaMemcpyAsync(c->f_buf[c->cur], c->pin_f32, sizeof(float) * n, cudaMemcpyHostToDevice,
                                     c->stream));
        }
    }
    int save = 0;
    unsigned long long idx = 0;
    DTB_TRY(enqueue_step(c, t_start, t_stop, &dt, &save, verbose, &idx));
    if (c->prec == DTB_F64)
        DTB_CUDA(cudaMemcpyAsync(f_out, c->f_buf[c->cur], sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    else
        DTB_CUDA(cudaMemcpyAsync(c->pin_f32, c->f_buf[c->cur], sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    const bool want_diag = verbose == 1 || verbose == 2 || verbose == 3 || diag_out;
    if (want_diag)
        DTB_CUDA(cudaMemcpyAsync(c->pin_hist, c->hist + idx, sizeof(StepDiagDev), cudaMemcpyDeviceToHost, c->stream));
    DTB_TRY(check_kernel_err(c));  // the one wait of the round trip
    if (c->prec == DTB_F32)
        for (size_t k = 0; k < n; ++k) f_out[k] = c->pin_f32[k];
    if (dt_out) *dt_out = dt;
    if (save_out) *save_out = save;
    if (diag_out) std::memcpy(diag_out, c->pin_hist, sizeof(StepDiagDev));
    return DTB_OK;
}

int32_t dtb_prepare(dtb_ctx* c) {
    DTB_RANGE("dtb_prepare");
    DTB_CHECK(c, DTB_EINVAL, "dtb_prepare: null context");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    if (c->prec == DTB_MIXED) return batch_prepare(c);
    if (c->profiling) return DTB_OK;  // profiled runs launch step by step
    DTB_TRY(ensure_graph(c, 0));
    DTB_CUDA(cudaGraphUpload(c->graph, c->stream));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    return DTB_OK;
}

int32_t dtb_run(dtb_ctx* c, const double* dt_scales, int64_t nsteps, int32_t verbose, dtb_step_diag* diag_hist) {
    DTB_RANGE("dtb_run");
    DTB_CHECK(c && (dt_scales || nsteps == 0), DTB_EINVAL, "dtb_run: null argument");
    DTB_CHECK(nsteps >= 0, DTB_EINVAL, "dtb_run: nsteps < 0");
    DTB_CHECK(c->prec != DTB_MIXED, DTB_ESTATE, "dtb_run: batched contexts use the dtb_batch_* entry points");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    for (int64_t s0 = 0; s0 < nsteps; s0 += c->hist_cap) {
        const int64_t n = std::min<int64_t>(c->hist_cap, nsteps - s0);
        DTB_CUDA(cudaStreamSynchronize(c->stream));  // pinned staging is reused
        std::memcpy(c->pin_dt, dt_scales + s0, sizeof(double) * (size_t)n);
        DTB_TRY(run_chunk(c, n, verbose, true));
        c->steps_run += n;
        if (diag_hist) {
            DTB_CUDA(cudaMemcpyAsync(c->pin_hist, c->hist, sizeof(StepDiagDev) * (size_t)n, cudaMemcpyDeviceToHost,
                                     c->stream));
            DTB_TRY(check_kernel_err(c));
            std::memcpy(diag_hist + s0, c->pin_hist, sizeof(StepDiagDev) * (size_t)n);
        }
    }
    if (c->profiling) DTB_TRY(flush_profile(c));
    if (!diag_hist) DTB_TRY(check_kernel_err(c));
    return DTB_OK;
}

int32_t dtb_solve_schedule(double dt_initial, const double* t_save, int64_t n_save, double dt0, int32_t precision,
                           int64_t* steps_per_interval, double* dt_scales, int64_t cap, int64_t* n_total_out) {
    DTB_CHECK(t_save && n_save >= 1, DTB_EINVAL, "dtb_solve_schedule: need t_save");
    DTB_CHECK(dt_initial > 0 && std::isfinite(dt_initial), DTB_EINVAL, "dtb_solve_schedule: dt must be > 0");
    const double d0 = precision == DTB_F32 ? (double)(float)dt0 : dt0;
    double dt = dt_initial;
    int64_t total = 0;
    for (int64_t i = 1; i < n_save; ++i) {
        double t_start = t_save[i - 1];
        const double t_stop = t_save[i];
        int64_t k = 0;
        bool save = false;
        while (!save) {  // Solver.jl:34-37 with SteppingMethods.jl:18-23
            if (t_start + dt >= t_stop) {
                dt = t_stop - t_start;
                save = true;
            }
            if (dt_scales && total < cap) dt_scales[total] = dt / d0;
            ++total;
            ++k;
            t_start += dt;
            DTB_CHECK(total <= kMaxScheduleSteps, DTB_EINVAL,
                      "dtb_solve_schedule: more than 1e8 steps; the truncated dt of a save point is carried "
                      "into later intervals (Solver.jl:35) and has become too small (dt = " +
                          std::to_string(dt) + ")");
        }
        if (steps_per_interval) steps_per_interval[i - 1] = k;
    }
    if (n_total_out) *n_total_out = total;
    return DTB_OK;
}

int32_t dtb_get_f(dtb_ctx* c, double* f) {
    DTB_CHECK(c && f, DTB_EINVAL, "dtb_get_f: null argument");
    DTB_CHECK(c->prec != DTB_MIXED, DTB_ESTATE, "dtb_get_f: batched contexts use the dtb_batch_* entry points");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    if (c->prec == DTB_F64) {
        DTB_CUDA(cudaMemcpyAsync(f, c->f_buf[c->cur], sizeof(double) * (size_t)c->n_state, cudaMemcpyDeviceToHost,
                                 c->stream));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
    } else {
        DTB_CUDA(cudaMemcpyAsync(c->pin_f32, c->f_buf[c->cur], sizeof(float) * (size_t)c->n_state,
                                 cudaMemcpyDeviceToHost, c->stream));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
        for (int64_t i = 0; i < c->n_state; ++i) f[i] = c->pin_f32[i];
    }
    return DTB_OK;
}

int32_t dtb_set_f(dtb_ctx* c, const double* f) {
    DTB_CHECK(c && f, DTB_EINVAL, "dtb_set_f: null argument");
    DTB_CHECK(c->prec != DTB_MIXED, DTB_ESTATE, "dtb_set_f: batched contexts use the dtb_batch_* entry points");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    if (c->prec == DTB_F64) {
        DTB_CUDA(cudaMemcpyAsync(c->f_buf[c->cur], f, sizeof(double) * (size_t)c->n_state, cudaMemcpyHostToDevice,
                                 c->stream));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
    } else {
        DTB_CUDA(cudaStreamSynchronize(c->stream));  // the staging buffer may still feed a copy
        for (int64_t i = 0; i < c->n_state; ++i) c->pin_f32[i] = (float)f[i];
        DTB_CUDA(cudaMemcpyAsync(c->f_buf[c->cur], c->pin_f32, sizeof(float) * (size_t)c->n_state,
                                 cudaMemcpyHostToDevice, c->stream));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
    }
    return DTB_OK;
}

int32_t dtb_reset(dtb_ctx* c) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_reset: null context");
    DTB_CHECK(c->prec != DTB_MIXED, DTB_ESTATE, "dtb_reset: batched contexts use the dtb_batch_* entry points");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    DTB_CUDA(cudaMemcpyAsync(c->f_buf[c->cur], c->f_init_dev, c->esz * (size_t)c->n_state, cudaMemcpyDeviceToDevice,
                             c->stream));
    return DTB_OK;
}

int32_t dtb_solve(dtb_ctx* c, double dt_initial, const double* t_save, int64_t n_save, int32_t verbose, double* f_out,
                  int64_t* n_steps_out) {
    DTB_CHECK(c && t_save && f_out && n_save >= 1, DTB_EINVAL, "dtb_solve: null argument");
    return dtb_solve_ex(c, dt_initial, t_save, n_save, verbose, f_out, nullptr, nullptr, nullptr, n_steps_out);
}

}  // extern "C"

// ------------------------------------------------------------------ pipelined Solve
// Solver.jl:1-64 without a host round trip per save interval: the step schedule depends only
// on dt and t_save, so it is generated on the host chunk by chunk (up to hist_cap steps, dt
// staging double-buffered) and every chunk's steps are enqueued at once. At a save point the
// state is copied on the device into a ring slot (and its moments computed there), and the
// copy stream moves the slot to pinned memory while the next interval steps; the host copies
// a slot out only when the ring wraps or at the end.
constexpr int kSaveRing = 4;

static int ensure_pipe(dtb_ctx* c) {
    if (c->pipe_ready) return DTB_OK;
    const size_t fb = c->esz * (size_t)c->n_state;
    DTB_CUDA(cudaMallocHost(&c->pin_dt2, sizeof(double) * 2 * (size_t)c->hist_cap));
    DTB_CUDA(cudaMallocHost(&c->save_pin, fb * kSaveRing));
    DTB_TRY(c->alloc(&c->save_dev, fb * kSaveRing));
    DTB_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 4 + 2 * kSaveRing; ++k) DTB_CUDA(cudaEventCreateWithFlags(&c->pipe_ev[k], cudaEventDisableTiming));
    c->pipe_ready = true;
    return DTB_OK;
}

// n steps through the device counter from its current value (graph replays where they fit).
static int run_steps(dtb_ctx* c, int64_t n, int verbose) {
    int64_t done = 0;
    if (!c->profiling && n >= c->graph_steps) {
        if (c->cur != 0) {
            DTB_TRY(run_loose(c, 1, verbose, false));
            done++;
        }
        while (n - done >= c->graph_steps) {
            DTB_CUDA(cudaGraphLaunch(c->graph, c->stream));
            done += c->graph_steps;
            c->host_ctr += c->graph_steps;
            c->launches += c->graph_launches;
        }
    }
    return run_loose(c, n - done, verbose, c->profiling);
}

namespace {
struct StepInfo {
    double t, dt, t_stop;
};
}  // namespace

extern "C" int32_t dtb_solve_ex(dtb_ctx* c, double dt_initial, const double* t_save, int64_t n_save, int32_t verbose,
                                double* f_out, const double* w, double* number, double* energy,
                                int64_t* n_steps_out) {
    DTB_RANGE("dtb_solve");
    DTB_CHECK(c && t_save && n_save >= 1, DTB_EINVAL, "dtb_solve_ex: null argument");
    DTB_CHECK(!w || (number && energy), DTB_EINVAL, "dtb_solve_ex: moments need number and energy outputs");
    DTB_CHECK(c->prec != DTB_MIXED, DTB_ESTATE, "dtb_solve: batched contexts use the dtb_batch_* entry points");
    DTB_CHECK(dt_initial > 0 && std::isfinite(dt_initial), DTB_EINVAL, "dtb_solve: dt must be > 0");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    DTB_TRY(ensure_pipe(c));
    const bool want_diag = verbose == 1 || verbose == 2 || verbose == 3;
    if (want_diag && !c->pin_hist2)
        DTB_CUDA(cudaMallocHost(&c->pin_hist2, sizeof(StepDiagDev) * 2 * (size_t)c->hist_cap));
    if (!c->profiling) DTB_TRY(ensure_graph(c, verbose));
    const size_t fb = c->esz * (size_t)c->n_state;
    const size_t mstride = (size_t)2 * c->ns * c->n_space;
    double* mom_all = nullptr;
    if (w) {
        DTB_CUDA(cudaMemcpyAsync(c->mom_w, w, sizeof(double) * (size_t)c->n_mom, cudaMemcpyHostToDevice, c->stream));
        DTB_CUDA(cudaMallocAsync(&mom_all, sizeof(double) * mstride * (size_t)n_save, c->stream));
    }
    cudaEvent_t* ev_dt = c->pipe_ev;
    cudaEvent_t* ev_hist = c->pipe_ev + 2;
    cudaEvent_t* ev_saved = c->pipe_ev + 4;
    cudaEvent_t* ev_landed = c->pipe_ev + 4 + kSaveRing;
    int64_t owner[kSaveRing];
    for (auto& o : owner) o = -1;
    int rc = DTB_OK;

    auto drain = [&](int sl) -> int {
        if (owner[sl] < 0) return DTB_OK;
        DTB_CUDA(cudaEventSynchronize(ev_landed[sl]));
        double* dst = f_out + (size_t)owner[sl] * c->n_state;
        const char* src = static_cast<const char*>(c->save_pin) + fb * sl;
        if (c->prec == DTB_F64) {
            std::memcpy(dst, src, fb);
        } else {
            const float* s32 = reinterpret_cast<const float*>(src);
            for (int64_t k = 0; k < c->n_state; ++k) dst[k] = s32[k];
        }
        owner[sl] = -1;
        return DTB_OK;
    };
    int64_t save_idx = 0;
    auto save = [&]() -> int {
        if (f_out) {
            const int sl = (int)(save_idx % kSaveRing);
            DTB_TRY(drain(sl));
            void* dslot = static_cast<char*>(c->save_dev) + fb * sl;
            DTB_CUDA(cudaMemcpyAsync(dslot, c->f_buf[c->cur], fb, cudaMemcpyDeviceToDevice, c->stream));
            DTB_CUDA(cudaEventRecord(ev_saved[sl], c->stream));
            DTB_CUDA(cudaStreamWaitEvent(c->copy_stream, ev_saved[sl], 0));
            DTB_CUDA(cudaMemcpyAsync(static_cast<char*>(c->save_pin) + fb * sl, dslot, fb, cudaMemcpyDeviceToHost,
                                     c->copy_stream));
            DTB_CUDA(cudaEventRecord(ev_landed[sl], c->copy_stream));
            owner[sl] = save_idx;
        }
        if (w) {
            double* out = mom_all + mstride * (size_t)save_idx;
            if (c->prec == DTB_F64)
                DTB_CUDA(launch_moments_f64(reinterpret_cast<const double*>(c->f_buf[c->cur]), (int)c->n_mom,
                                            c->n_space, c->sp_off_dev, c->ns, c->mom_w, out, c->stream));
            else
                DTB_CUDA(launch_moments_f32(reinterpret_cast<const float*>(c->f_buf[c->cur]), (int)c->n_mom,
                                            c->n_space, c->sp_off_dev, c->ns, c->mom_w, out, c->stream));
        }
        ++save_idx;
        return DTB_OK;
    };
    std::vector<StepInfo> info[2];
    bool pending[2] = {false, false};
    int64_t pending_n[2] = {0, 0};
    auto print_chunk = [&](int b) -> int {
        if (!pending[b]) return DTB_OK;
        DTB_CUDA(cudaEventSynchronize(ev_hist[b]));
        const StepDiagDev* h = c->pin_hist2 + (size_t)b * c->hist_cap;
        for (int64_t k = 0; k < pending_n[b]; ++k) print_cr(verbose, h[k], info[b][k].t, info[b][k].t_stop, info[b][k].dt);
        pending[b] = false;
        return DTB_OK;
    };

    // Solver.jl:22 reset; :14 the initial state is the first save
    rc = dtb_reset(c);
    if (rc == DTB_OK) rc = save();
    const double d0 = dt0_eff(c);
    double dt = dt_initial;
    int64_t interval = 1, total = 0;
    double t_start = t_save[0];
    int b = 0;
    std::vector<int64_t> marks;
    while (rc == DTB_OK && interval < n_save) {
        // the staging buffer of two chunks ago is free once its upload has run
        if ((rc = cudaEventSynchronize(ev_dt[b]) == cudaSuccess ? DTB_OK : DTB_ECUDA) != DTB_OK) break;
        if ((rc = print_chunk(b)) != DTB_OK) break;
        double* stage = c->pin_dt2 + (size_t)b * c->hist_cap;
        info[b].clear();
        marks.clear();
        int64_t n = 0;
        while (n < c->hist_cap && interval < n_save) {  // Solver.jl:25-37 with SteppingMethods.jl:18-23
            const double t_stop = t_save[interval];
            bool at_save = false;
            if (t_start + dt >= t_stop) {
                dt = t_stop - t_start;
                at_save = true;
            }
            stage[n] = dt / d0;
            if (want_diag) info[b].push_back({t_start, dt, t_stop});
            t_start += dt;
            ++n;
            if (++total > kMaxScheduleSteps) {
                set_error("dtb_solve: more than 1e8 steps; the truncated dt of a save point is carried into later "
                          "intervals (Solver.jl:35) and has become too small");
                rc = DTB_EINVAL;
                break;
            }
            if (at_save) {
                marks.push_back(n);
                ++interval;
                t_start = t_save[interval - 1];
            }
        }
        if (rc != DTB_OK) break;
        DTB_CUDA(cudaMemcpyAsync(c->dt_arr, stage, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
        DTB_CUDA(cudaEventRecord(ev_dt[b], c->stream));
        DTB_CUDA(cudaMemsetAsync(c->ctr, 0, sizeof(unsigned long long), c->stream));
        c->host_ctr = 0;
        int64_t done = 0;
        for (int64_t mk : marks) {
            if ((rc = run_steps(c, mk - done, verbose)) != DTB_OK) break;
            done = mk;
            if ((rc = save()) != DTB_OK) break;
        }
        if (rc == DTB_OK && done < n) rc = run_steps(c, n - done, verbose);
        if (rc != DTB_OK) break;
        if (want_diag) {
            DTB_CUDA(cudaMemcpyAsync(c->pin_hist2 + (size_t)b * c->hist_cap, c->hist, sizeof(StepDiagDev) * (size_t)n,
                                     cudaMemcpyDeviceToHost, c->stream));
            DTB_CUDA(cudaEventRecord(ev_hist[b], c->stream));
            pending[b] = true;
            pending_n[b] = n;
        }
        b ^= 1;
    }
    // finish: diagnostics of the last two chunks in order, the save ring, the moments
    cudaError_t e1 = cudaStreamSynchronize(c->stream);
    cudaError_t e2 = cudaStreamSynchronize(c->copy_stream);
    if (rc == DTB_OK && e1 != cudaSuccess) rc = (set_error(std::string("CUDA error: ") + cudaGetErrorString(e1)), DTB_ECUDA);
    if (rc == DTB_OK && e2 != cudaSuccess) rc = (set_error(std::string("CUDA error: ") + cudaGetErrorString(e2)), DTB_ECUDA);
    if (rc == DTB_OK) rc = print_chunk(b);
    if (rc == DTB_OK) rc = print_chunk(b ^ 1);
    for (int64_t k = std::max<int64_t>(0, save_idx - kSaveRing); rc == DTB_OK && k < save_idx; ++k)
        rc = drain((int)(k % kSaveRing));
    if (w) {
        if (rc == DTB_OK) {
            std::vector<double> hm(mstride * (size_t)n_save);
            cudaError_t e = cudaMemcpyAsync(hm.data(), mom_all, sizeof(double) * hm.size(), cudaMemcpyDeviceToHost,
                                            c->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
            if (e != cudaSuccess) {
                set_error(std::string("CUDA error: ") + cudaGetErrorString(e));
                rc = DTB_ECUDA;
            } else {
                for (size_t k = 0; k < hm.size() / 2; ++k) {
                    number[k] = hm[2 * k];
                    energy[k] = hm[2 * k + 1];
                }
            }
        }
        cudaFreeAsync(mom_all, c->stream);
        cudaStreamSynchronize(c->stream);
    }
    if (rc != DTB_OK) return rc;
    DTB_TRY(check_kernel_err(c));
    c->steps_run += total;
    if (n_steps_out) *n_steps_out = total;
    return DTB_OK;
}

extern "C" {

int32_t dtb_moments(dtb_ctx* c, const double* w, double* number, double* energy) {
    DTB_CHECK(c && w && number && energy, DTB_EINVAL, "dtb_moments: null argument");
    DTB_CHECK(c->prec != DTB_MIXED, DTB_ESTATE, "dtb_moments: batched contexts use the dtb_batch_* entry points");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    DTB_CUDA(cudaMemcpyAsync(c->mom_w, w, sizeof(double) * (size_t)c->n_mom, cudaMemcpyHostToDevice, c->stream));
    if (c->prec == DTB_F64)
        DTB_CUDA(launch_moments_f64(reinterpret_cast<const double*>(c->f_buf[c->cur]), (int)c->n_mom, c->n_space,
                                    c->sp_off_dev, c->ns, c->mom_w, c->mom_out, c->stream));
    else
        DTB_CUDA(launch_moments_f32(reinterpret_cast<const float*>(c->f_buf[c->cur]), (int)c->n_mom, c->n_space,
                                    c->sp_off_dev, c->ns, c->mom_w, c->mom_out, c->stream));
    std::vector<double> out((size_t)2 * c->ns * c->n_space);
    DTB_CUDA(cudaMemcpyAsync(out.data(), c->mom_out, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, c->stream));
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < out.size() / 2; ++k) {
        number[k] = out[2 * k];
        energy[k] = out[2 * k + 1];
    }
    return DTB_OK;
}

int32_t dtb_device_bytes(dtb_ctx* c, int64_t* bytes) {
    DTB_CHECK(c && bytes, DTB_EINVAL, "dtb_device_bytes: null argument");
    *bytes = (int64_t)c->dev_bytes;
    return DTB_OK;
}

int32_t dtb_get_stream(dtb_ctx* c, void** stream) {
    DTB_CHECK(c && stream, DTB_EINVAL, "dtb_get_stream: null argument");
    *stream = c->stream;
    return DTB_OK;
}

int32_t dtb_sync(dtb_ctx* c) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_sync: null context");
    DeviceGuard g(c->device);
    DTB_CUDA(cudaStreamSynchronize(c->stream));
    if (c->committed) DTB_TRY(check_kernel_err(c));
    return DTB_OK;
}

int32_t dtb_launches_per_step(dtb_ctx* c, int32_t* n) {
    DTB_CHECK(c && n, DTB_EINVAL, "dtb_launches_per_step: null argument");
    DTB_TRY(dtb_commit(c));
    *n = (c->n_units > 0 && c->n_bin_cells > 0 ? 2 : 1) + (c->symplectic ? 1 : 0);
    return DTB_OK;
}

int32_t dtb_launch_count(dtb_ctx* c, int64_t* n) {
    DTB_CHECK(c && n, DTB_EINVAL, "dtb_launch_count: null argument");
    *n = c->launches;
    return DTB_OK;
}

int32_t dtb_set_profiling(dtb_ctx* c, int32_t on) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_set_profiling: null context");
    if (c->profiling && c->prof_pending) DTB_TRY(flush_profile(c));
    c->profiling = on != 0;
    c->prof_ms = 0.0;
    c->prof_n = 0;
    c->prof_pending = 0;
    return DTB_OK;
}

int32_t dtb_selftest_bounded_wait(dtb_ctx* c, double limit_s) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_selftest_bounded_wait: null context");
    DTB_CHECK(limit_s > 0 && limit_s <= 2.0, DTB_EINVAL, "dtb_selftest_bounded_wait: limit must be in (0, 2] s");
    DTB_TRY(dtb_commit(c));
    DeviceGuard g(c->device);
    DTB_CUDA(launch_bounded_wait_selftest((unsigned long long)(limit_s * 1e9), c->err, c->stream));
    if (c->prec == DTB_MIXED) {
        DTB_CUDA(cudaMemcpyAsync(c->pin_err, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        DTB_CUDA(cudaStreamSynchronize(c->stream));
        if (*c->pin_err) {
            cudaMemsetAsync(c->err, 0, sizeof(int), c->stream);
            cudaStreamSynchronize(c->stream);
            set_error("a bounded device wait gave up (self-test)");
            return DTB_ETIMEOUT;
        }
        return DTB_OK;
    }
    const int rc = check_kernel_err(c);
    if (rc == DTB_ETIMEOUT) set_error("a bounded device wait gave up (self-test)");
    return rc;
}

int32_t dtb_gain_kernel_stats(dtb_ctx* c, double* avg_ms, double* bytes_per_launch) {
    DTB_CHECK(c, DTB_EINVAL, "dtb_gain_kernel_stats: null context");
    DTB_TRY(dtb_commit(c));
    if (bytes_per_launch) *bytes_per_launch = c->gain_bytes * c->n_bin_cells;
    if (avg_ms) *avg_ms = c->prof_n ? c->prof_ms / (double)c->prof_n : 0.0;
    return DTB_OK;
}

}  // extern "C"
