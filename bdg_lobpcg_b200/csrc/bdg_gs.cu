// bdg_gs.cu -- ground-state producer on the GPU (real psi0).
//
// The BdG path needs a stationary condensate psi0 and its chemical potential
// mu.  The reference takes psi0 from a file (src/io.c:13-50); this module
// computes it on the device with the same FFT pass kernels as the operators:
//
//   split-step (Strang) imaginary-time propagation
//     psi <- F^-1[e^{-dt k^2/4} F psi]
//     psi <- psi * exp(-dt (V + g |psi|^2 + g_dd Phi[|psi|^2]))
//     psi <- F^-1[e^{-dt k^2/4} F psi],  normalised to sum |psi|^2 dV = 1
//   until the per-step change of mu = <psi|H|psi> is below tol, then
//   bordered Newton steps on F(psi, mu) = H(psi) psi - mu psi with the
//   normalisation constraint (the Jacobian of F is the BdG operator M; each
//   step solves M a = r, M b = psi by CG on the device) to remove the
//   O(dt^2) splitting error, so that K psi0 = 0 to rounding.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include "bdg_dev.h"

__global__ void k_potential_step(double *__restrict__ psi, const double *__restrict__ V, const double *__restrict__ phi,
                                 double g, double dt, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double p = psi[i];
    const double u = V[i] + g * p * p + (phi ? phi[i] : 0.0);
    psi[i] = p * exp(-dt * u);
  }
}

// Hpsi = kin + (V + g psi^2 + phi) psi
__global__ void k_apply_h(const double *__restrict__ psi, const double *__restrict__ kin, const double *__restrict__ V,
                          const double *__restrict__ phi, double g, double *__restrict__ Hpsi, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double p = psi[i];
    Hpsi[i] = kin[i] + (V[i] + g * p * p + (phi ? phi[i] : 0.0)) * p;
  }
}

// ltM = V + 3 g psi^2 + phi - mu (the M local term of this psi), ltK = ltM
__global__ void k_local_m(const double *__restrict__ psi, const double *__restrict__ V, const double *__restrict__ phi,
                          double g, double mu, double *__restrict__ ltM, double *__restrict__ ltK, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double p = psi[i];
    const double base = V[i] + g * p * p + (phi ? phi[i] : 0.0) - mu;
    ltK[i] = base;
    ltM[i] = base + 2.0 * g * p * p;
  }
}

#define GS_CK(x)                                                              \
  do {                                                                        \
    cudaError_t _e = (x);                                                     \
    if (_e != cudaSuccess) return bdgd_check(_e, #x);                         \
  } while (0)
#define GS_BL(x)                                                              \
  do {                                                                        \
    if ((x) != CUBLAS_STATUS_SUCCESS) {                                       \
      bdgd_set_error("cuBLAS failure in %s", #x);                             \
      return BDGD_ERR_CUDA;                                                   \
    }                                                                         \
  } while (0)

struct GsState {
  bdgd_ctx *c;
  cublasHandle_t h;
  double *V, *psi, *t1, *t2, *phi;
  long long S;
  double g, dV;
  bool dip;
};

static int gs_grid(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b > 4096 ? 4096 : b);
}

static int gs_normalize(GsState &s) {
  double nrm = 0;
  GS_BL(cublasDnrm2(s.h, (int)s.S, s.psi, 1, &nrm));
  const double sc = 1.0 / (nrm * sqrt(s.dV));
  GS_BL(cublasDscal(s.h, (int)s.S, &sc, s.psi, 1));
  return BDGD_OK;
}

// Hpsi into t2 (uses t1, phi), returns mu
static int gs_mu(GsState &s, double *mu) {
  bdgd_ctx *c = s.c;
  int rc = bdgd_apply(c, BDGD_OP_KINETIC, BDGD_F64, s.psi, s.S, s.t1, s.S, 1);
  if (rc) return rc;
  if (s.dip && (rc = bdgd_run_internal(c, 102, s.psi, s.S, s.phi, s.S, 1))) return rc;
  bdgd_count_launch();
  k_apply_h<<<gs_grid(s.S), 256, 0, c->stream>>>(s.psi, s.t1, s.V, s.dip ? s.phi : nullptr, s.g, s.t2, s.S);
  GS_CK(cudaGetLastError());
  double a = 0, b = 0;
  GS_BL(cublasDdot(s.h, (int)s.S, s.psi, 1, s.t2, 1, &a));
  GS_BL(cublasDdot(s.h, (int)s.S, s.psi, 1, s.psi, 1, &b));
  *mu = a / b;
  return BDGD_OK;
}

// x = M^-1 b by CG (M of the fields currently on the context)
static int gs_cg(GsState &s, const double *b, double *x, double *r, double *p, double *q) {
  bdgd_ctx *c = s.c;
  const int n = (int)s.S;
  GS_CK(cudaMemsetAsync(x, 0, sizeof(double) * s.S, c->stream));
  GS_CK(cudaMemcpyAsync(r, b, sizeof(double) * s.S, cudaMemcpyDeviceToDevice, c->stream));
  GS_CK(cudaMemcpyAsync(p, b, sizeof(double) * s.S, cudaMemcpyDeviceToDevice, c->stream));
  double rr = 0;
  GS_BL(cublasDdot(s.h, n, r, 1, r, 1, &rr));
  const double bn = sqrt(rr);
  for (int it = 0; it < 20000 && sqrt(rr) > 1e-14 * bn; ++it) {
    int rc = bdgd_apply(c, BDGD_OP_M, BDGD_F64, p, s.S, q, s.S, 1);
    if (rc) return rc;
    double pq = 0;
    GS_BL(cublasDdot(s.h, n, p, 1, q, 1, &pq));
    const double al = rr / pq, nal = -al;
    GS_BL(cublasDaxpy(s.h, n, &al, p, 1, x, 1));
    GS_BL(cublasDaxpy(s.h, n, &nal, q, 1, r, 1));
    double rn = 0;
    GS_BL(cublasDdot(s.h, n, r, 1, r, 1, &rn));
    const double be = rn / rr, one = 1.0;
    GS_BL(cublasDscal(s.h, n, &be, p, 1));
    GS_BL(cublasDaxpy(s.h, n, &one, r, 1, p, 1));
    rr = rn;
  }
  return BDGD_OK;
}

extern "C" int bdgd_ground_state(bdgd_ctx *c, const double *V_host, double g, double dt, double tol, int max_steps,
                                 int newton_steps, double *psi_inout, double *mu_out, int *steps_out,
                                 double *stationarity_out) {
  if (c->cplx) {
    bdgd_set_error("bdgd_ground_state: real wavefunctions only");
    return BDGD_ERR_UNSUPPORTED;
  }
  GsState s;
  s.c = c;
  s.S = c->S;
  s.g = g;
  s.dV = (c->L[0] / c->N[0]) * (c->dim > 1 ? c->L[1] / c->N[1] : 1.0) * (c->dim > 2 ? c->L[2] / c->N[2] : 1.0);
  s.dip = c->dipolar && c->vdd && c->dim == 3;
  double *buf = nullptr;
  GS_CK(cudaMalloc(&buf, sizeof(double) * s.S * 9));
  s.V = buf;
  s.psi = buf + s.S;
  s.t1 = buf + 2 * s.S;
  s.t2 = buf + 3 * s.S;
  s.phi = buf + 4 * s.S;
  double *a = buf + 5 * s.S, *bv = buf + 6 * s.S, *r = buf + 7 * s.S, *pq = buf + 8 * s.S;
  int rc = BDGD_OK;
  if (cublasCreate(&s.h) != CUBLAS_STATUS_SUCCESS) {
    cudaFree(buf);
    bdgd_set_error("cublasCreate failed");
    return BDGD_ERR_CUDA;
  }
  cublasSetStream(s.h, c->stream);
  double mu = 0, mu_old = 0;
  int steps = 0;
  do {
    GS_CK(cudaMemcpyAsync(s.V, V_host, sizeof(double) * s.S, cudaMemcpyHostToDevice, c->stream));
    GS_CK(cudaMemcpyAsync(s.psi, psi_inout, sizeof(double) * s.S, cudaMemcpyHostToDevice, c->stream));
    if ((rc = gs_normalize(s))) break;
    if ((rc = gs_mu(s, &mu_old))) break;
    c->kin_dt = 0.25 * dt;
    for (steps = 1; steps <= max_steps; ++steps) {
      if ((rc = bdgd_run_internal(c, 101, s.psi, s.S, s.t1, s.S, 1))) break;
      if (s.dip && (rc = bdgd_run_internal(c, 102, s.t1, s.S, s.phi, s.S, 1))) break;
      bdgd_count_launch();
      k_potential_step<<<gs_grid(s.S), 256, 0, c->stream>>>(s.t1, s.V, s.dip ? s.phi : nullptr, g, dt, s.S);
      if ((rc = bdgd_run_internal(c, 101, s.t1, s.S, s.psi, s.S, 1))) break;
      if ((rc = gs_normalize(s))) break;
      if ((rc = gs_mu(s, &mu))) break;
      const double d = fabs(mu - mu_old);
      mu_old = mu;
      if (d < tol) break;
    }
    if (rc) break;
    if (steps > max_steps) steps = max_steps;
    // Newton polish: r = H psi - mu psi (t2 holds H psi after gs_mu)
    double res = 0;
    for (int nt = 0; nt <= newton_steps; ++nt) {
      if ((rc = gs_mu(s, &mu))) break;
      const double nmu = -mu;
      GS_CK(cudaMemcpyAsync(r, s.t2, sizeof(double) * s.S, cudaMemcpyDeviceToDevice, c->stream));
      GS_BL(cublasDaxpy(s.h, (int)s.S, &nmu, s.psi, 1, r, 1));
      double rn = 0;
      GS_BL(cublasDnrm2(s.h, (int)s.S, r, 1, &rn));
      res = rn * sqrt(s.dV);
      if (nt == newton_steps || res < 1e-13) break;
      // fields of M for this psi: wavefunction, local terms
      if (!c->ltM64) GS_CK(cudaMalloc((void **)&c->ltM64, sizeof(double) * s.S));
      if (!c->ltK64) GS_CK(cudaMalloc((void **)&c->ltK64, sizeof(double) * s.S));
      if (!c->wf64) GS_CK(cudaMalloc(&c->wf64, sizeof(double) * s.S));
      GS_CK(cudaMemcpyAsync(c->wf64, s.psi, sizeof(double) * s.S, cudaMemcpyDeviceToDevice, c->stream));
      bdgd_count_launch();
      k_local_m<<<gs_grid(s.S), 256, 0, c->stream>>>(s.psi, s.V, s.dip ? s.phi : nullptr, g, mu, c->ltM64, c->ltK64,
                                                     s.S);
      GS_CK(cudaGetLastError());
      c->has_wf = 1;
      if ((rc = gs_cg(s, r, a, s.t1, s.t2, pq))) break;
      if ((rc = gs_cg(s, s.psi, bv, s.t1, s.t2, pq))) break;
      double pa = 0, pb = 0;
      GS_BL(cublasDdot(s.h, (int)s.S, s.psi, 1, a, 1, &pa));
      GS_BL(cublasDdot(s.h, (int)s.S, s.psi, 1, bv, 1, &pb));
      const double dmu = pa / pb, mone = -1.0;
      GS_BL(cublasDaxpy(s.h, (int)s.S, &mone, a, 1, s.psi, 1));
      GS_BL(cublasDaxpy(s.h, (int)s.S, &dmu, bv, 1, s.psi, 1));
      if ((rc = gs_normalize(s))) break;
    }
    if (rc) break;
    GS_CK(cudaMemcpyAsync(psi_inout, s.psi, sizeof(double) * s.S, cudaMemcpyDeviceToHost, c->stream));
    GS_CK(cudaStreamSynchronize(c->stream));
    *mu_out = mu;
    *steps_out = steps;
    *stationarity_out = res;
  } while (0);
  cublasDestroy(s.h);
  cudaFree(buf);
  c->kin_dt = 0.0;
  return rc;
}
