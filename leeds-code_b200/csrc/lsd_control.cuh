// lsd_control.cuh -- the predictor/corrector control of the main loop (timestep.F90
// tim_check_cgce :744-830, tim_new_tstep :837-870; main.F90:100-164), written once for
// the host (lsd_corrector / lsd_predictor used one at a time, and the C-ABI mirror
// lsd_tim_check_cgce) and for the device (the control kernels of the one-graph step).
#pragma once

#include <cmath>

// The module variables of timestep.F90 that the loop control reads and writes.
struct PcState {
  double t;        // tim_t
  double dt;       // tim_dt
  double dterr;    // tim_dterr (accumulated over the corrector's fields, reset after a check)
  double corr_dt;  // tim_corr_dt
  double lasterr;  // lasterr of tim_check_cgce (a saved local there)
  double cfl_dt;   // tim_cfl_dt of the last evaluation (non_maxtstep)
  int it;          // tim_it: 0 = the next evaluation starts a step, k = corrector k follows
  int step;        // tim_step
  int pcn;         // tim_pcn: fixed corrector count (control 2), -1 = off
  int pad_;
};

// The parameters of the control (parameters.F90 d_timestep, d_dterr, d_courant,
// d_corr_upper, d_corr_lower, i_time_step_control).
struct PcParams {
  double timestep, dterr, courant, corr_upper, corr_lower;
  int control;
  int pad_;
};

// tim_check_cgce (timestep.F90:744-830) after a corrector whose norm is c.dterr.
// Returns false when the reference gives up (it then ends the run: tim_step =
// i_maxtstep - 1): dt -> 0, more than 10 iterations, or a growing error above the limit.
// c.it becomes 0 when the step is complete, c.it + 1 when another corrector follows.
__host__ __device__ inline bool pc_check_cgce(PcState& c, const PcParams& p) {
  bool ok = true;
  const double dterr = c.dterr;
  if (p.control == 1) {
    if (c.it == 1) { c.corr_dt = dterr; c.lasterr = 1e99; }
    if (c.dt < 1e-12 && c.step > 30) { c.it = 0; ok = false; }
    else if (c.it > 10) { c.it = 0; ok = false; }
    else if (dterr > c.lasterr) { if (dterr > 1.0) ok = false; c.it = 0; }
    else if (dterr > 1.0) { c.lasterr = dterr; c.it = c.it + 1; }
    else c.it = 0;
  } else {
    if (c.it == 1) { c.corr_dt = c.dt * sqrt(p.dterr / dterr); c.lasterr = 1e99; }
    if (c.dt < 1e-12 && c.step > 30) { c.it = 0; ok = false; }
    else if (c.it == c.pcn) c.it = 0;
    else if (c.it > 10) { c.it = 0; ok = false; }
    else if (dterr > c.lasterr) {
      if (dterr > 2.0 * p.dterr) ok = false;
      if (dterr < 2.0 * p.dterr) c.corr_dt = c.dt / (1e1 * p.courant);
      c.it = 0;
    } else if (dterr > p.dterr) { c.lasterr = dterr; c.it = c.it + 1; }
    else c.it = 0;
  }
  c.dterr = 0.0;
  return ok;
}

// tim_new_tstep (timestep.F90:837-870) with the CFL limit c.cfl_dt of the evaluation just
// done: the dt of the next step; returns true (tim_new_dt) when it differs from c.dt by
// more than 3 %, in which case c.dt takes it and the operators must be rebuilt.
__host__ __device__ inline bool pc_new_tstep(PcState& c, const PcParams& p) {
  double dt = c.dt;
  if (p.control == 1) {
    if (c.corr_dt > p.corr_upper) dt = 0.5 * dt;
    if (c.corr_dt < p.corr_lower) dt = 1.273974 * dt;
    if (c.step == 0) dt = fmin(dt / 1e3, 1e-8);
  } else {
    if (c.corr_dt > 0.0) dt = fmin(c.corr_dt, dt * 2.0 / p.courant);
    if (c.cfl_dt > 0.0) dt = fmin(c.cfl_dt, dt);
    if (c.step == 0) dt = fmin(dt / 1e3, 1e-10);
    dt = dt * p.courant;
  }
  if (dt < c.dt * 0.97 || dt > c.dt * 1.03) {
    c.dt = dt;
    return true;
  }
  return false;
}

// The device-resident control block of one context during lsd_step: the state above, the
// counters of the call, and its outcome.
struct PcDev {
  PcState s;
  double last_dterr;    // the norm of the last corrector
  int nsteps;           // steps asked of this call
  int steps_left;       // of this call
  int steps_done, correctors, evaluations, rebuilds;
  int status;           // LSD_OK, or the failure that ended the call
  int iters;            // corrector iterations of the current step (hard cap, see k_pc_corr)
  int loops;            // step-loop iterations of this call (hard cap, see k_pc_end)
};
