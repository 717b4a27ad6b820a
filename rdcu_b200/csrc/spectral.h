// Fused pseudospectral RHS of the dictionary: plan and launchers.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "internal.h"

namespace rdcu {

// A coupling term as the reference stores it (rdcu.cu:606,654-660): coefficient and
// the integer list (field, Yidx, pow, Yidx, pow, ...).
struct HostTerm {
  double C;
  std::vector<int> ints;
};

// Where the inputs of one RHS evaluation come from and where f goes.
struct RhsIO {
  int mode = 0;               // 0: plain y -> f;  1: DP45 stage (buffers resolved on device)
  int stage = 0;              // mode 1: 1 (k1 = f(y)) or 2..7
  const double* y = nullptr;  // mode 0 input
  double* f = nullptr;        // mode 0 output
  DP45Bufs bufs{};            // mode 1
  DP45Ctl* ctl = nullptr;     // mode 1
  double* err_part = nullptr; // mode 1, stage 7: per-CTA partial sums of err^2
  double* ytemp_out = nullptr;// mode 1, stages >= 2: write the stage state here instead of its slot
  // mode 1, stage 7 of an adaptive step (plans with wants_err_aux()): nN doubles the
  // forward pass fills with each point's slope sum sum_{j != 2, 7} e_j k_j, which the
  // inverse pass completes with e_7 k_7 (and divides by the scale atol + rtol
  // max(|y|, |y_new|), from y and the stage state it reads) instead of reading five
  // slopes again
  double* err_aux = nullptr;
};

struct PassCfg {
  int grid = 0, block = 0;
  size_t smem = 0;
  int per_cta = 0;  // pairs / rows / columns per CTA
};

// Caller-provided device memory for a plan (bump allocation, never freed by the plan).
struct PlanArena {
  char* base = nullptr;
  size_t size = 0;
  size_t used = 0;
  cudaStream_t stream = nullptr;  // table uploads are ordered on this stream
};

class SpectralBatch;

class SpectralPlan {
  friend class SpectralBatch;

 public:
  // Builds the plan; returns false with msg set when the problem is unsupported.
  bool init(int n, int ndim, const int* Ns, const double* Ls, const std::vector<HostTerm>& terms,
            std::string* msg);
  // A linear operator instead of a dictionary: output channel c = sum over its entries
  // of coef * multiplier(op) applied to input field src (coefficients unscaled).
  bool init_linear(int n_in, int ndim, const int* Ns, const double* Ls,
                   const std::vector<std::vector<ChanEntry>>& channels, std::string* msg);
  // out[c*N + point] = channel c of the linear operator applied to in (n_in fields).
  cudaError_t run_linear(const double* in, double* out, cudaStream_t stream);
  // New coefficients C[term] for the dictionary (same structure as at init).
  cudaError_t set_coefficients(const std::vector<double>& C);
  // Same plan with every device buffer carved from `arena` instead of cudaMalloc.
  bool init_in_arena(int n, int ndim, const int* Ns, const double* Ls, const std::vector<HostTerm>& terms,
                     PlanArena* arena, std::string* msg);
  void release();
  ~SpectralPlan() { release(); }

  // f = RHS(y) on `stream` (mode 0) or one DP45 stage (mode 1).  A DP45 stage may also
  // do the forward x pass of the stage after it (next, when fused is given): *fused
  // tells whether it did; the run of that next stage then passes fwd_done = true.
  cudaError_t run(const RhsIO& io, cudaStream_t stream, const RhsIO* next = nullptr, bool fwd_done = false,
                  bool* fused = nullptr);
  // All complex Y blocks (Y.dat layout) of y, written to Yout (device).
  cudaError_t run_Y(const double* y, double* Yout, cudaStream_t stream);

  struct PassTime {
    const char* name;
    double ms;
    double bytes;
  };
  // Times every pass of one RHS evaluation (io) `reps` times each.
  // With next (the stage after io), also the fused inverse/forward pass of the two.
  cudaError_t profile(const RhsIO& io, int reps, cudaStream_t stream, std::vector<PassTime>* out,
                      const RhsIO* next = nullptr);

  // FFT-only plan for the BDF preconditioner: z = (I + alpha*J_lin)^-1 r with J_lin
  // the constant-coefficient linear FD operator of `lin` (solved mode by mode).
  bool init_precond(int n, int ndim, const int* Ns, const double* Ls, const std::vector<LinEntry>& lin,
                    std::string* msg);
  cudaError_t precond(const double* r, double* z, double alpha, cudaStream_t stream);
  // the same with alpha read on the device from alpha_dev (captured solves)
  cudaError_t precond(const double* r, double* z, double alpha, const double* alpha_dev, cudaStream_t stream);

  int n = 0, ndim = 0, Ns[3] = {1, 1, 1};
  double Ls[3] = {1, 1, 1};
  long long N = 0;  // grid points
  int M = 0, Mh = 0, R = 0;
  int nch = 0;                // channels of the hot RHS
  int nparts_max = 0;         // error partials buffer size needed (stage-7 epilogue)
  size_t device_bytes = 0;
  // Whether stage 7 of an adaptive step should carry RhsIO::err_aux (the x pass one row
  // per warp evaluates the error from it).
  bool wants_err_aux() const { return inv_row_; }
  // Nonzero when a pass on TMA tiles gave up waiting for its copies (read and cleared).
  int take_pipe_error();
  // Incremented whenever a device buffer that launches capture is replaced (work
  // captured in a CUDA graph before that must be captured again).
  int buffers_gen = 0;

 private:
  bool built_ = false;
  // line plans: x axis (length M) and the strided axes (0..ndim-2)
  LinePlan plan_x_{}, plan_ax_[3]{};
  double2* tw_x_ = nullptr;
  double2* tw_ax_[3] = {nullptr, nullptr, nullptr};
  double* kv_ = nullptr;
  int kv_off_[3] = {0, 0, 0};
  // hot-path channels and dictionary
  int* ch_off_ = nullptr;
  ChanEntry* ch_ent_ = nullptr;
  ChanEntry* ch_sorted_ = nullptr;  // hot entries in operator order (mid pass fast path)
  DictTerm* d_terms_ = nullptr;
  DictFactor* d_fac_ = nullptr;
  int* d_field_begin_ = nullptr;
  int* d_fold_ = nullptr;
  double* d_poly_ = nullptr;        // dense polynomial form of the dictionary (DictTable.poly)
  int poly_nf_ = 0, poly_count_ = 0;
  std::vector<int> h_poly_mono_;    // monomial of each dictionary term (dense form)
  int nterms_dict_ = 0;
  int nfac_dict_ = 0;
  int kv_total_ = 0;
  std::vector<int> h_ch_off_, h_ych_off_;  // host copies of the channel offsets
  // Y-mode channels (every block, real and imaginary part)
  int ych_ = 0;
  int* ych_off_ = nullptr;
  ChanEntry* ych_ent_ = nullptr;
  int* ych_dst_ = nullptr;
  // preconditioner tables
  LinEntry* lin_ent_ = nullptr;
  int nlin_ = 0;
  double* sinv_ = nullptr;
  double* cosv_ = nullptr;
  int sc_off_[3] = {0, 0, 0};
  PassCfg midsolve_{};
  // spectral buffers
  double2* Sf_ = nullptr;  // field half spectra [n][R][Mh]
  double2* Sc_ = nullptr;  // channel half spectra [max(nch, G)][R][Mh]
  int sc_rows_ = 0;        // channel capacity of Sc_
  PlanArena* arena_ = nullptr;
  const std::vector<std::vector<ChanEntry>>* explicit_channels_ = nullptr;
  std::vector<ChanEntry> h_ch_ent_;
  std::vector<int> h_ent_term_;   // term index of each hot entry (-1: not a term coefficient)
  std::vector<DictTerm> h_dterms_;
  std::vector<int> h_dict_term_;  // term index of each dictionary term
  double inv_n_ = 1.0;
  template <typename T>
  cudaError_t dev_alloc(T** p, size_t bytes);
  template <typename T>
  cudaError_t upload_vec(T** dst, const std::vector<T>& v);
  // launch configurations
  PassCfg fwd_, inv_, mid_[2], c2c_f_, c2c_i_, mult_;
  // 3D passes on TMA tiles (k_mid_pipe, k_c2c_pipe) and the warp-per-row x pass
  // (k_inv_row): tensor maps of the field and channel spectra, operator groups and
  // their coefficient matrices, error word
  bool pipe_mid_ = false, pipe_c2c_ = false, inv_row_ = false;
  int pipe_grid_ = 0, mid_ngrp_ = 0, sms_ = 1;
  CUtensorMap tm_sf_{}, tm_sc_{}, tm_sf_c2c_{}, tm_sc_c2c_{};
  ChanEntry* mid_grp_ = nullptr;
  double* mid_A_ = nullptr;
  bool mid_tab_ = false;           // multiplier tables (no group mixes axis 0 with another axis)
  double2* mid_mz_ = nullptr;      // [L0][nch][n]
  double2* mid_mc_ = nullptr;      // [N1 * Mh][nch][n]
  bool mid2_ = false;              // k_mid_pipe2: at most two groups on axis 0 alone
  bool mid_real_ = false;          // every multiplier of the tables is real
  bool mid_tables_built_ = false;
  int mid_nz_ = 0;                 // their number
  double* mid_bz_ = nullptr;       // [max(1, mid_nz_)][L0] beta_g(z)
  double2* mid_rz_ = nullptr;      // [max(1, mid_nz_)][nch][n] i^q A_g
  std::vector<double> h_kv_;       // host copy of the wavenumbers
  cudaError_t build_mid_tables(const std::vector<ChanEntry>& grp, const std::vector<double>& A);
  int* pipe_err_ = nullptr;
  void setup_pipes();
  bool encode_sc_map();
  cudaError_t launch_mid_pipe(const RhsIO& io, cudaStream_t stream);
  // rev: tiles from the last to the first (-1: the inverse pass does, the forward pass not)
  cudaError_t launch_c2c_pipe(bool inv, int nplanes, cudaStream_t stream, const RhsIO& io, int rev = -1);
  cudaError_t launch_inv_row(const RhsIO& io, cudaStream_t stream);
  // stage io's inverse x pass fused with stage next's forward x pass (k_inv_fwd_row)
  bool fuse_rows_ = false;
  bool fuse_ok(const RhsIO& io, const RhsIO& next) const;
  cudaError_t launch_inv_fwd_row(const RhsIO& io, const RhsIO& next, cudaStream_t stream);
  // 3D x passes that also transform along axis 1, one thread-block cluster per plane
  // (k_fwd_plane, k_inv_plane): enabled flags and persistent grid sizes
  bool plane_fwd_ = false, plane_inv_ = false;
  int plane_fwd_grid_ = 0, plane_inv_grid_ = 0;
  void setup_planes();
  bool plane_fwd_ok(const RhsIO& io) const;
  bool plane_inv_ok(const RhsIO& io) const;
  cudaError_t launch_plane_fwd(const RhsIO& io, cudaStream_t stream);
  cudaError_t launch_plane_inv(const RhsIO& io, cudaStream_t stream);

  ChanTable chan_table(const int* off, const ChanEntry* ent, int nch) const;
  DictTable dict_table() const;
  cudaError_t launch_passes(const RhsIO& io, const ChanTable& ct, const std::vector<int>& hoff, int nch_run,
                            int g_first, double* Yout, const int* ydst, cudaStream_t stream, int yplain = 0,
                            const RhsIO* next = nullptr, bool* fused = nullptr);
  size_t dict_smem_bytes() const;
  cudaError_t launch_forward(const double* y, cudaStream_t stream);
  bool geometry(std::string* msg);
  cudaError_t ensure_channel_capacity(int rows);
  std::vector<double> poly_table() const;  // dense coefficients from h_dterms_
};

// One problem of a batch: a 2D plan and its DP45 state.
struct BatchMember {
  SpectralPlan* plan = nullptr;
  DP45Bufs bufs{};
  DP45Ctl* ctl = nullptr;
  double* err_part = nullptr;  // one partial per grid row (stage 7)
};

// DP45 stages of many 2D problems of different sizes and coefficients: every pass is one
// persistent launch over a list of (problem, tile) work items; each item runs the CTA
// body of the single-problem kernel with that problem's arguments.  Nothing a pass
// computes depends on the tiling (the error partials are per grid row), so results are
// bitwise those of each problem's own plan while the tiles are chosen for the batch.
class SpectralBatch {
 public:
  // elems: target complex values per CTA of the x passes and of the axis-0 pass
  bool init(const std::vector<BatchMember>& members, int elems, std::string* msg);
  void release();
  ~SpectralBatch() { release(); }
  // stage 1 (k1 = f(y)) .. 7 of every running member, 3 launches
  cudaError_t launch_stage(int stage, cudaStream_t stream);
  size_t device_bytes = 0;
  int elems = 0;
  int nitems[3] = {0, 0, 0};  // work items of the fwd_x, mid and inv_x passes

 private:
  struct Impl;
  Impl* impl_ = nullptr;
};

}  // namespace rdcu
