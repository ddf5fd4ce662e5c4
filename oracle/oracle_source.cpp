// oracle_source.cpp -- source-particle creation of the reference (one rank,
// thermal "surface-like" source in every shell), restated on the CPU.
// TEST INFRASTRUCTURE ONLY: makes the input particles of parity cases and of
// the CPU baseline.
//
// SOURCE/sourceenergy.f90:3-55, SOURCE/sourcenumbers.f90:3-171 (nmpi = 1),
// SOURCE/vacancies.f90:3-30, SOURCE/interior_source.f90:3-172,
// SOURCE/source_transformdirection.f90:3-47, transportmod.f:129-145.
#include <cstring>
#include "oracle_internal.h"

using namespace orc;

extern "C" {

// sourceenergy.f90:21-29 (surface source, renormalised to L_bol)
void orc_sourceenergy(int nx, const double* xarr, const double* radtemp, double L_bol,
                      double* emit, double* tot_sthermal) {
  double s = 0.0;
  for (int i = 0; i < nx; ++i) {
    double rcell = (xarr[i + 1] + xarr[i]) / 2.0;  // grid_setup.f:46
    emit[i] = pc_pi * pc_c * sq(rcell) * pc_acoef * pow4(radtemp[i]);
  }
  for (int i = 0; i < nx; ++i) s = s + emit[i];
  for (int i = 0; i < nx; ++i) emit[i] = emit[i] / s * L_bol;
  double t = 0.0;
  for (int i = 0; i < nx; ++i) t = t + emit[i];
  *tot_sthermal = t;
}

// sourcenumbers.f90:3-94 for a single rank without surface source.
int64_t orc_sourcenumbers(int nx, const double* emit, double pwr, int64_t src_ns, int64_t nvacant,
                          int32_t* nvol) {
  for (int l = 0; l < nx; ++l) nvol[l] = 0;
  const int64_t nstot = src_ns;
  double etot = 0.0;
  for (int l = 0; l < nx; ++l) etot = etot + std::pow(emit[l], pwr);
  etot = etot + std::pow(0.0, pwr);  // tot_esurf**pwr
  int64_t ncactive = 0;
  for (int l = 0; l < nx; ++l) ncactive += emit[l] > 0.0;
  if (nvacant < ncactive) return -1;
  const int64_t nsavail = nstot;
  double edone = 0.0;
  int64_t ndone = 0;
  const double invn = 1.0 / (double)nsavail;
  double einv = 1.0 / etot;
  if (etot == 0.0) einv = 0.0;
  for (int l = 0; l < nx; ++l) {
    double en = std::pow(emit[l], pwr);
    if (en == 0.0) continue;
    int64_t n = (int64_t)(en * (double)nsavail * einv);
    if (n < 1) n = 1;
    if (edone * einv > (double)ndone * invn) n = n + 1;
    nvol[l] = (int32_t)n;
    edone = edone + en;
    ndone = ndone + n;
  }
  if (ndone == 0) return -2;
  int64_t sum = 0;
  for (int l = 0; l < nx; ++l) sum += nvol[l];
  int64_t nextra = nstot - sum;
  if (nextra > nx) return -3;
  const int64_t nsmean = nstot / ncactive;
  while (nextra != 0) {
    for (int l = 0; l < nx; ++l) {
      if (nextra == 0) break;
      if (nvol[l] < nsmean) continue;
      int s = nextra > 0 ? 1 : -1;
      nvol[l] += s;
      nextra -= s;
    }
  }
  int64_t nnew = 0;
  for (int l = 0; l < nx; ++l)
    if (emit[l] != 0.0) nnew += nvol[l];
  return nnew;
}

// vacancies.f90 + interior_source.f90 + source_transformdirection.f90 with the
// single non-threaded mzran stream rnd_state.  Returns 0 or an error code.
int orc_interior_source(int nx, int ng, const double* xarr, const double* vxarr,
                        const double* wlinv, const double* radtemp, const double* emit, double pwr,
                        const int32_t* nvol, int64_t npart, orc_packet* prt, int32_t* isvacant,
                        orc_rnd* state, int rngmode, uint64_t seed) {
  int64_t nnew = 0;
  for (int l = 0; l < nx; ++l)
    if (emit[l] != 0.0) nnew += nvol[l];
  if (nnew > npart) return 1;
  std::vector<int64_t> ivacant;
  ivacant.reserve(nnew);
  for (int64_t ip = 0; ip < npart && (int64_t)ivacant.size() < nnew; ++ip)
    if (isvacant[ip]) ivacant.push_back(ip);
  if ((int64_t)ivacant.size() < nnew) return 2;
  std::vector<double> emitprob(ng);
  int64_t ipart = 0;
  auto X = [&](int i) { return xarr[i - 1]; };
  for (int i = 1; i <= nx; ++i) {
    const int l = i;
    if (std::pow(emit[l - 1], pwr) == 0.0) continue;
    const int nemit = nvol[l - 1];
    const int nhere = nvol[l - 1];
    if (nhere < 1) continue;
    const double tradinv = 1.0 / radtemp[l - 1];
    orc_specintv(tradinv, wlinv, ng, ng, 1, 0, emitprob.data());
    double s = 0.0;
    for (int g = 0; g < ng; ++g) s = s + emitprob[g];
    for (int g = 0; g < ng; ++g) emitprob[g] = emitprob[g] / s;
    const int icnb1 = i - 1 > 1 ? i - 1 : 1;
    const int icnb2 = i + 1 < nx ? i + 1 : nx;
    for (int ii = 1; ii <= nhere; ++ii) {
      const int64_t ivac = ivacant[ipart];
      orc_packet& p = prt[ivac];
      isvacant[ivac] = 0;
      ipart++;
      // rngmode 0: the single mzran stream rnd_state; 1: Philox stream
      // (seed, pid = slot, stream 1) shared with the GPU source kernel
      uint32_t kdraw = 0;
      auto mzran_real = [&](orc_rnd* st) {
        return rngmode == 0 ? orc::mzran_real(st) : orc::philox_real(seed, (uint64_t)ivac, 1u, kdraw++);
      };
      double denom2 = 0.0;
      double r1 = mzran_real(state);
      int iig = 1;
      for (int ig = 1; ig <= ng; ++ig) {
        iig = ig;
        if (r1 >= denom2 && r1 < denom2 + emitprob[ig - 1]) break;
        denom2 = denom2 + emitprob[ig - 1];
      }
      r1 = mzran_real(state);
      p.wl = 1.0 / ((1.0 - r1) * wlinv[iig - 1] + r1 * wlinv[iig]);
      const double ep0 = emit[l - 1] / (double)nemit;
      p.e = ep0;
      p.e0 = ep0;
      r1 = mzran_real(state);
      p.mu = std::sqrt(r1);
      r1 = mzran_real(state);
      p.om = pc_pi2 * r1;
      double r3 = 0.0, r2 = 1.0, x0 = 0.0;
      double uul = 0.5 * (emit[icnb1 - 1] + emit[l - 1]);
      double uur = 0.5 * (emit[icnb2 - 1] + emit[l - 1]);
      double uumax = uul > uur ? uul : uur;
      uul = uul / uumax;
      uur = uur / uumax;
      while (r2 > r3) {
        r1 = mzran_real(state);
        x0 = std::pow(r1 * cube(X(i + 1)) + (1.0 - r1) * cube(X(i)), third_r4);
        r3 = (x0 - X(i)) / (X(i + 1) - X(i));
        r3 = r3 * uur + (1.0 - r3) * uul;
        r2 = mzran_real(state);
      }
      p.x = x0;
      p.y = -1.0;  // grd_yarr(1) of a 1-D grid (inputstrmod.f:202)
      p.z = 0.0;
    }
  }
  // source_transformdirection.f90:20-44 with direction2lab1
  for (int64_t k = 0; k < nnew; ++k) {
    orc_packet& p = prt[ivacant[k]];
    int ix = orc::binsrch(p.x, xarr, nx + 1, false);
    double vx = (vxarr[ix - 1] * (xarr[ix] - p.x) + vxarr[ix] * (p.x - xarr[ix - 1])) /
                (xarr[ix] - xarr[ix - 1]);
    double cmffact = 1.0 + p.mu * vx * cinv;
    double mu = (p.mu + vx * cinv) / cmffact;
    mu = mu < 1.0 ? mu : 1.0;
    mu = mu > -1.0 ? mu : -1.0;
    p.mu = mu;
  }
  return 0;
}

}  // extern "C"
