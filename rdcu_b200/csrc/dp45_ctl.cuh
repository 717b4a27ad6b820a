// Device-side DP45 step control shared by the single-problem engine and the ensemble.
#pragma once
#include <cuda_runtime.h>

#include "internal.h"

namespace rdcu {

constexpr int kCtlThreads = 256;

// k_dp45_arm's state reset for one problem
__device__ __forceinline__ void dp45_arm(DP45Ctl* c, int check, double t1, double hmin, double hmax, int eval_i,
                                         int n_eval, int max_attempts) {
  c->check_t1 = check;
  c->t1 = t1;
  c->hmin = hmin;
  c->hmax = hmax;
  c->eval_i = eval_i;
  c->n_eval = n_eval;
  c->max_attempts = max_attempts;
  c->attempts_this_launch = 0;
  c->log_count = 0;
  c->stop_reason = kStopNone;
  c->running = check ? ((c->t < t1 && c->h > hmin) ? 1 : 0) : 1;
  if (!c->running) c->stop_reason = kStopDone;
}

// One controller update after an attempt, by a block of kCtlThreads threads: the sum of
// the stage-7 error partials in a fixed order, then (thread 0) dp45_step's accept/reject
// logic (dp45.cu:109-146), slot rotation, attempt log and stop test.  log_cap == 0
// disables the log (and its stop reason).
__device__ __forceinline__ void dp45_control(DP45Ctl* c, const double* part, double* log_h, double* log_t,
                                             int* log_acc, double nN, const double* t_eval) {
  if (!c->running) return;
  __shared__ double red[kCtlThreads];
  const int tid = threadIdx.x;
  double s = 0.0;
  if (!c->fixed) {
    // unrolled so that a thread's loads are in flight together; the sum keeps its order
    const int np = c->nparts;
#pragma unroll 16
    for (int i = tid; i < np; i += kCtlThreads) s += part[i];
  }
  red[tid] = s;
  __syncthreads();
  for (int w = kCtlThreads / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid != 0) return;
  double t = c->t, h = c->h;
  int acc;
  if (c->fixed) {
    acc = 1;
    c->t_last = t;
    t = t + h;
  } else {
    // dp45.cu:117-146: RMS norm of the scaled error, factor 0.9 err^-1/5 (0.2 if NaN)
    double norm = sqrt(red[0]);
    norm /= pow(nN, 0.5);
    c->err_norm = norm;
    double factor = 0.9 * pow(norm, -0.2);
    if (isnan(factor)) factor = 0.2;
    if (norm < 1) {
      acc = 1;
      c->t_last = t;
      t = t + h;
      if (factor > 10) factor = 10;
      h *= factor;
      if (h > c->hmax) h = c->hmax;
    } else {
      acc = 0;
      if (factor < 1) {
        if (factor < 0.2) factor = 0.2;
        h *= factor;
      }
    }
  }
  if (acc) {
    const int y_old = c->y_slot, yn = c->yn_slot, yl = c->yl_slot;
    c->yl_slot = y_old;
    c->y_slot = yn;
    c->yn_slot = yl;
    c->last_k1_buf = c->k1_buf;
    c->last_k7_buf = c->k7_buf;
    const int k1 = c->k1_buf;
    c->k1_buf = c->k7_buf;
    c->k7_buf = k1;
    c->n_accepted++;
  }
  c->t = t;
  c->h = h;
  c->accepted = acc;
  c->n_attempts++;
  c->attempts_this_launch++;
  if (c->log_count < c->log_cap) {
    log_h[c->log_count] = h;
    log_t[c->log_count] = t;
    log_acc[c->log_count] = acc;
  }
  c->log_count++;
  if (!c->check_t1) {
    c->running = 0;
    return;
  }
  int reason = kStopNone;
  if (acc && c->eval_i < c->n_eval && t >= t_eval[c->eval_i]) reason = kStopOutput;
  else if (!(t < c->t1 && h > c->hmin)) reason = kStopDone;
  else if (c->log_cap > 0 && c->log_count >= c->log_cap) reason = kStopLog;
  else if (c->attempts_this_launch >= c->max_attempts) reason = kStopChunk;
  if (reason != kStopNone) {
    c->running = 0;
    c->stop_reason = reason;
  }
}

}  // namespace rdcu
