// Timing driver around the UNMODIFIED GPU prior art of the reference (dynex.cu).
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile into oracle/_ref/libdynex_gpu_ref.so
// with the reference source included verbatim from its read-only location (the recipe
// passes its path as DYNEX_GPU_REF_SRC; nothing of it is copied into this repository).  The
// reference's own main() is renamed so that this file can load one formula into the
// reference's globals and device buffers and run the reference's own kernels:
//   gpu_step        dynex.cu:327-428   (one thread per clause, CAS-loop double atomics)
//   gpu_euler       dynex.cu:261-292   (Euler step, clamps, changed-variable count)
//   gpu_reset_dxdt  dynex.cu:303-311,  gpu_reset_vars  dynex.cu:295-300
// The host loop of solveGPU (dynex.cu:432-619: per step the three kernels, device-to-host
// reads of loc and energy, then the adaptive trials with a device-to-host read of the
// changed-variable count after each, then the final Euler kernel) is restated in
// refgpu_run() below, in the same order of launches and copies, without its screen output
// and with a step cap, so that a fixed number of the reference's GPU steps can be timed.
// The reference GPU code differs from dynex.cc in its arithmetic (atomics in arbitrary
// order, its own step-size rule); it is timed here, never used as the oracle.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>

#define main dynex_gpu_main
#include DYNEX_GPU_REF_SRC
#undef main

namespace {
bool g_gpu_ready = false;

void free_gpu() {
  if (!g_gpu_ready) return;
  cudaFree(d_x);
  cudaFree(d_x_tmp);
  cudaFree(d_dxdt);
  cudaFree(d_cls);
  cudaFree(d_clauseSizes);
  cudaFree(d_loc);
  cudaFree(d_varchanges);
  cudaFree(d_energy);
  free(cls);
  free(clauseSizes);
  cls = nullptr;
  clauseSizes = nullptr;
  g_gpu_ready = false;
}
}  // namespace

extern "C" {

// Loads one formula (flat signed literals, clause i = lits[clause_off[i] .. clause_off[i+1]),
// at most max_lits_system = 10 literals per clause, dynex.cu:150) into the reference's globals
// and device buffers as its main() does (dynex.cu:938-939, 1025-1034), with the parameters
// alpha beta gamma delta epsilon zeta and the Xl bound factor.  Returns 0, or -1 for a clause
// that is too long or a CUDA error.
int refgpu_setup(int nv, int mc, const int* lits, const long long* clause_off,
                 const double* params, int xl_max_factor) {
  free_gpu();
  n = nv;
  m = mc;
  cls = (int*)calloc((size_t)m * max_lits_system, sizeof(int));
  clauseSizes = (int*)calloc((size_t)m, sizeof(int));
  for (int i = 0; i < m; i++) {
    const long long b = clause_off[i], e = clause_off[i + 1];
    if (e - b > max_lits_system) return -1;
    clauseSizes[i] = (int)(e - b);
    for (long long j = b; j < e; j++) cls[(size_t)i * max_lits_system + (j - b)] = lits[j];
  }
  dmm_alpha = params[0];
  dmm_beta = params[1];
  dmm_gamma = params[2];
  dmm_delta = params[3];
  dmm_epsilon = params[4];
  dmm_zeta = params[5];
  xl_max = xl_max_factor;
  xl_max = xl_max * m;
  if (xl_max <= 0) xl_max = INT_MAX;
  const size_t N = (size_t)n + 2 * (size_t)m;
  if (cudaMalloc(&d_x, N * sizeof(TFloat)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_x_tmp, N * sizeof(TFloat)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_dxdt, N * sizeof(TFloat)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_cls, (size_t)m * max_lits_system * sizeof(int)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_clauseSizes, (size_t)m * sizeof(int)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_loc, sizeof(int)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_varchanges, sizeof(int)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_energy, sizeof(float)) != cudaSuccess) return -1;
  cudaMemcpy(d_cls, cls, (size_t)m * max_lits_system * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(d_clauseSizes, clauseSizes, (size_t)m * sizeof(int), cudaMemcpyHostToDevice);
  g_gpu_ready = true;
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

void refgpu_teardown(void) { free_gpu(); }

// Uploads x0 (n + 2m doubles) and runs up to max_steps steps of solveGPU's loop
// (dynex.cu:472-568), stopping early when the right-hand side reports loc == 0.
// *wall_ms: host wall time of the steps (the loop synchronizes with the device at every
// copy); *steps_done, *last_loc: steps taken and the last unsatisfied count.
int refgpu_run(const double* x0, int max_steps, double* wall_ms, int* steps_done, int* last_loc) {
  if (!g_gpu_ready) return -1;
  const int N = n + 2 * m;
  const int tpb = 256;
  const int grid_all = (N + tpb - 1) / tpb;
  const int grid_m = (m + tpb - 1) / tpb;
  if (cudaMemcpy(d_x, x0, (size_t)N * sizeof(TFloat), cudaMemcpyHostToDevice) != cudaSuccess)
    return -1;
  cudaDeviceSynchronize();
  int steps = 0;
  TFloat t = 0.0;
  double h = 0.125;
  const auto t0 = std::chrono::steady_clock::now();
  gpu_reset_vars<<<1, 1>>>(d_loc, d_energy, d_varchanges, m);
  while (steps < max_steps) {
    gpu_reset_dxdt<<<grid_all, tpb>>>(d_dxdt, N);
    gpu_reset_vars<<<1, 1>>>(d_loc, d_energy, d_varchanges, m);
    gpu_step<<<grid_m, tpb>>>(d_x, d_dxdt, d_cls, d_loc, d_energy, m, n, xl_max, dmm_alpha,
                              dmm_beta, dmm_gamma, dmm_delta, dmm_epsilon, dmm_zeta,
                              d_clauseSizes);
    cudaMemcpy(h_loc, d_loc, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(h_energy, d_energy, sizeof(float), cudaMemcpyDeviceToHost);
    if (h_loc[0] == 0) break;
    t = t + h;
    bool accepted = false;
    const double h_min = 0.0078125;
    h = 0.125;
    while (!accepted) {
      gpu_reset_vars<<<1, 1>>>(d_loc, d_energy, d_varchanges, m);
      gpu_euler<<<grid_all, tpb>>>(d_x_tmp, d_x, d_dxdt, N, t, h, n, m, xl_max, d_varchanges);
      cudaMemcpy(h_varchanges, d_varchanges, sizeof(int), cudaMemcpyDeviceToHost);
      if (h_varchanges[0] == 0) accepted = true;
      h = h * 1 / 2;
      if (h <= h_min) {
        h = h_min;
        accepted = true;
      }
    }
    gpu_euler<<<grid_all, tpb>>>(d_x, d_x, d_dxdt, N, t, h, n, m, xl_max, d_varchanges);
    steps++;
  }
  const cudaError_t e = cudaDeviceSynchronize();
  const auto t1 = std::chrono::steady_clock::now();
  *wall_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  *steps_done = steps;
  *last_loc = h_loc[0];
  return e == cudaSuccess ? 0 : -1;
}

}  // extern "C"
