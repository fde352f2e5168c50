/*
 * ymoracle — CPU restatement (plain C, FP64) of the reference's Wilson-flow
 * path.  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA kernels
 * and the "port" CPU baseline.  No product code links or calls it.
 *
 * Field layout everywhere in this file is the reference's .bin layout
 * (src/InputOutput/inputconf.cpp:114-155): site-major with x fastest,
 * site = x + Nx*(y + Ny*(z + Nz*t)); per site mu = 0..3; per link 18 doubles,
 * row-major 3x3, (re, im) interleaved (include/Math/su3.h:63).
 * Element k of link (site, mu) is U[(site*4 + mu)*18 + k].
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

int yo_version(void);

/* 3x3 complex algebra, reference term order (include/Math/su3.h:143-183, src/Math/su3.cpp:28-48). */
void yo_mul(const double* a, const double* b, double* c);
void yo_dag(const double* a, double* c);
/* e^{iQ} for Hermitian traceless Q by Cayley-Hamilton (src/Math/su3.cpp:96-183). */
void yo_exp(const double* q, double* r);
void yo_exp_many(const double* q, double* r, long n);

/* Z_mu for every site (src/Actions/puregauge.cpp:36-79).  Zmu: V x 18. */
void yo_derivative(const double* U, const int n[4], int mu, double* Zmu);
/* One Luscher RK3 step in place (src/Apps/wilsonflow.cpp:141-172).  Z: V x 4 x 18 scratch. */
void yo_flow_step(double* U, double* Z, const int n[4], double eps);
void yo_flow_stage(double* U, double* Z, const int n[4], double eps, int stage);
/* plaq, topc, energy exactly as SuperObs::compute (src/Observables/superobs.cpp:31-128). */
void yo_superobs(const double* U, const int n[4], double out[3]);
/* nsteps RK3 steps; rows (step, t, plaq, topc, energy) at step 0 and every `every` steps
 * (and the last step).  t accumulates as t += eps (src/Apps/wilsonflow.cpp:126).
 * table holds >= 5*(nsteps/every + 2) doubles; returns the row count. */
int yo_flow(double* U, const int n[4], double eps, int nsteps, int every, double* table);

/* Seeded synthetic fields (Philox4x32-10 keyed by seed and config id, counter =
 * global link index) — the generators of the parity fixtures. */
void yo_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void yo_gen_expiah(double* U, const int n[4], double a, uint64_t seed, uint32_t config);
void yo_gen_haar_mix(double* U, const int n[4], double frac, uint64_t seed, uint32_t config);
void yo_gen_cold(double* U, const int n[4]);
/* Metropolis restated from src/Apps/gaugefieldfactory.cpp:192-220 (the reference's
 * own generator does not compile); returns the acceptance ratio. */
double yo_gen_metropolis(double* U, const int n[4], double beta, double su3eps, int sweeps,
                         int hits, uint64_t seed);
/* The device generator's checkerboard chain with counter-based random numbers
 * (sweeps numbered from sweep0); returns the number of accepted proposals. */
long yo_gen_metropolis_cb(double* U, const int n[4], double beta, double su3eps, int sweeps, int hits,
                          uint64_t seed, uint32_t sweep0);
/* FP64 Gram-Schmidt reunitarisation of nlinks 18-double links in place. */
void yo_reunitarize(double* U, long nlinks);
/* max over links of |U U^+ - 1| and |det U - 1|. */
void yo_unitarity(const double* U, long nlinks, double out[2]);

#ifdef __cplusplus
}
#endif
