// The power spectrum of the mass assignment, measured on the forward FFT of
// each PM evaluation (the z pass bins |rho_k|^2 on the fly), and what the
// reference derives from it.
//
// Reference: CorrMeasure (Cosmos/Correlation.c:13-117), called by pmmain
// after the forward transform (Cosmos/pmmain.c:480-481): P(k) in bins of
// |k| in mode numbers, sigma_8 from the top-hat of radius 8 Mpc/h, the
// correlation function by the sine transform of P(k), and the log slope of
// xi between separations 2 and 3 cells.
#include <math.h>
#include <string.h>

#include <vector>

#include "ctx.cuh"

using namespace tpm;

extern "C" {

int tpm_set_power_spectrum(tpm_ctx *c, int enable) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  CK(cudaSetDevice(c->device));
  if (enable && !c->pk_acc) CK(dmalloc(c->arena, &c->pk_acc, sizeof(double) * 2 * (c->g.n + 1)));
  bool want = enable != 0;
  if (want != c->measure_pk) c->gen++;
  c->measure_pk = want;
  return 0;
}

int tpm_power_spectrum(tpm_ctx *c, double boxsize, double *pk, double *cor, int32_t nbins, double *sigma8,
                       double *slope) {
  if (!c || nbins < 0) return fail(TPM_E_ARG, "bad arguments to tpm_power_spectrum");
  if (!c->measure_pk || !(c->parts_valid & TPM_PART_PM))
    return fail(TPM_E_STATE, "no PM evaluation with the power spectrum enabled");
  CK(cudaSetDevice(c->device));
  const int nx = c->g.n;
  std::vector<double> acc(2 * (nx + 1));
  CK(cudaMemcpyAsync(acc.data(), c->pk_acc, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  std::vector<double> tpk(nx + 1), tcor(nx + 1, 0.0);
  for (int i = 0; i <= nx; i++) tpk[i] = acc[i];
  // bin averages and sigma_8 (Correlation.c:84-95)
  const double rng = nx;
  double rth = 8.0 / boxsize * nx;
  double std = 0;
  double fact = 2 * M_PI * rth / rng;
  for (int i = 1; i < nx + 1; i++) {
    double w = acc[nx + 1 + i];
    tpk[i] = w > 0 ? tpk[i] / w : 0.0;
    double thk = fact * i;
    std += tpk[i] * i * i * pow(sin(thk) - thk * cos(thk), 2.0) / pow(thk, 6.0);
  }
  std = sqrt(4 * M_PI * std * 9.0);
  // xi(r) at r = i cells by the sine transform (Correlation.c:96-102)
  for (int i = 1; i < nx + 1; i++) {
    double seper = 2 * M_PI * i / rng;
    for (int k = 1; k < nx + 1; k++) tcor[i] += sin(k * seper) * k * tpk[k];
    tcor[i] = (rng + rng) * tcor[i] / i;
  }
  double corn1 = 0;
  if (tcor[3] > 0 && tcor[2] > 0) corn1 = (log(tcor[3]) - log(tcor[2])) / (log(4.0) - log(3.0));
  int k = nbins < nx + 1 ? nbins : nx + 1;
  if (pk) memcpy(pk, tpk.data(), sizeof(double) * k);
  if (cor) memcpy(cor, tcor.data(), sizeof(double) * k);
  if (sigma8) *sigma8 = std;
  if (slope) *slope = corn1;
  return k;
}

}  // extern "C"
