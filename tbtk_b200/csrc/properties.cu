// The other properties of PropertyExtractor::ChebyshevExpander on the
// batched recursion: spin-polarized LDOS, density, magnetization and
// expectation values (Lib/src/PropertyExtractor/ChebyshevExpander.cpp
// :297-327,584-720).  The reference runs one recursion per (to, from) pair
// through calculateGreensFunction; here every pair a call needs is one
// target of one source of a single tbtkkpm_moments_batched call (one
// batched recursion on the device, damping included), the NonPrincipal
// Green's functions of all pairs come from one tbtkkpm_greens call (one
// energy-sum launch), and the host forms each property with the reference's
// expression and operation order, so FP64 results match the reference's bit
// for bit when the lookup table does.
#include "tbtkkpm.h"
#include "kpm_host.h"

#include <cmath>
#include <complex>
#include <vector>

namespace {

using cplx = std::complex<double>;

// G_NonPrincipal[k][e] of the pairs (to[k], from[owner[k]]) over the table's
// energies.
int greens_np(tbtkkpm_matrix *m, tbtkkpm_table *t, const std::vector<uint32_t> &from,
              const std::vector<uint32_t> &to, const std::vector<uint32_t> &owner,
              double broadening, int precision, std::vector<cplx> &G) {
  const uint32_t K = (uint32_t)to.size(), M = t->M;
  std::vector<cplx> mu((size_t)K * M);
  int rc = tbtkkpm_moments_batched(m, from.data(), (uint32_t)from.size(), to.data(), owner.data(),
                                   K, M, broadening, precision,
                                   reinterpret_cast<double *>(mu.data()), nullptr);
  if (rc) return rc;
  G.assign((size_t)K * t->E, cplx(0, 0));
  return tbtkkpm_greens(t, reinterpret_cast<const double *>(mu.data()), K, TBTKKPM_NONPRINCIPAL,
                        reinterpret_cast<double *>(G.data()));
}

// The four spin pairs of each site in the reference's order n = 0..3:
// to spin n/2, from spin n%2 (up-up, up-down, down-up, down-down); sources
// 2s (spin up) and 2s + 1 (spin down) of site s.
int spin_pairs(tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *up, const uint32_t *down,
               uint32_t S, double broadening, int precision, std::vector<cplx> &G) {
  std::vector<uint32_t> from(2 * (size_t)S), to(4 * (size_t)S), owner(4 * (size_t)S);
  for (uint32_t s = 0; s < S; s++) {
    from[2 * s] = up[s];
    from[2 * s + 1] = down[s];
    for (uint32_t n = 0; n < 4; n++) {
      to[4 * s + n] = n / 2 ? down[s] : up[s];
      owner[4 * s + n] = 2 * s + n % 2;
    }
  }
  return greens_np(m, t, from, to, owner, broadening, precision, G);
}

int check_common(tbtkkpm_matrix *m, tbtkkpm_table *t, const void *a, const void *b, uint32_t n,
                 const void *out, const char *fn) {
  if (!m || !t) return tbtkkpm::fail(TBTKKPM_ERR_ARGUMENT, "%s: NULL matrix or table", fn);
  if (n && (!a || !b || !out)) return tbtkkpm::fail(TBTKKPM_ERR_ARGUMENT, "%s: NULL pointer", fn);
  return TBTKKPM_OK;
}

}  // namespace

extern "C" int tbtkkpm_spin_polarized_ldos(tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *up,
                                           const uint32_t *down, uint32_t S, double broadening,
                                           int precision, double *out) {
  int rc = check_common(m, t, up, down, S, out, "spin_polarized_ldos");
  if (rc || S == 0) return rc;
  std::vector<cplx> G;
  if ((rc = spin_pairs(m, t, up, down, S, broadening, precision, G))) return rc;
  const uint32_t E = t->E;
  const cplx i(0, 1);
  cplx *o = reinterpret_cast<cplx *>(out);
  for (uint32_t s = 0; s < S; s++)
    for (uint32_t n = 0; n < 4; n++)
      for (uint32_t e = 0; e < E; e++) {
        // data[offset + e].at(n/2, n%2) += -i*G[e]/M_PI
        cplx v(0, 0);
        v += -i * G[(size_t)(4 * s + n) * E + e] / M_PI;
        o[((size_t)s * E + e) * 4 + n] = v;
      }
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_density(tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *sites, uint32_t S,
                               double broadening, int precision, const double *occupation, double dE,
                               double *out) {
  int rc = check_common(m, t, sites, occupation, S, out, "density");
  if (rc || S == 0) return rc;
  std::vector<uint32_t> from(sites, sites + S), to(sites, sites + S), owner(S);
  for (uint32_t s = 0; s < S; s++) owner[s] = s;
  std::vector<cplx> G;
  if ((rc = greens_np(m, t, from, to, owner, broadening, precision, G))) return rc;
  const uint32_t E = t->E;
  for (uint32_t s = 0; s < S; s++) {
    // data[offset] += weight*imag(G[e])/M_PI*dE
    double d = 0;
    for (uint32_t e = 0; e < E; e++) d += occupation[e] * std::imag(G[(size_t)s * E + e]) / M_PI * dE;
    out[s] = d;
  }
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_magnetization(tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *up,
                                     const uint32_t *down, uint32_t S, double broadening,
                                     int precision, const double *occupation, double dE,
                                     double *out) {
  int rc = check_common(m, t, up, down, S, out, "magnetization");
  if (!rc && S && !occupation) rc = tbtkkpm::fail(TBTKKPM_ERR_ARGUMENT, "magnetization: NULL occupation");
  if (rc || S == 0) return rc;
  std::vector<cplx> G;
  if ((rc = spin_pairs(m, t, up, down, S, broadening, precision, G))) return rc;
  const uint32_t E = t->E;
  const cplx i(0, 1);
  cplx *o = reinterpret_cast<cplx *>(out);
  for (uint32_t s = 0; s < S; s++)
    for (uint32_t n = 0; n < 4; n++) {
      // data[offset].at(n/2, n%2) += weight*(-i)*G[e]/M_PI*dE
      cplx v(0, 0);
      for (uint32_t e = 0; e < E; e++) v += occupation[e] * (-i) * G[(size_t)(4 * s + n) * E + e] / M_PI * dE;
      o[(size_t)s * 4 + n] = v;
    }
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_expectation_values(tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *to,
                                          const uint32_t *from, uint32_t P, double broadening,
                                          int precision, const double *occupation, double dE,
                                          double *out) {
  int rc = check_common(m, t, to, from, P, out, "expectation_values");
  if (!rc && P && !occupation) rc = tbtkkpm::fail(TBTKKPM_ERR_ARGUMENT, "expectation_values: NULL occupation");
  if (rc || P == 0) return rc;
  // distinct sources, each with the targets of its pairs
  std::vector<uint32_t> src, tgt(to, to + P), owner(P);
  for (uint32_t p = 0; p < P; p++) {
    uint32_t b = 0;
    while (b < src.size() && src[b] != from[p]) b++;
    if (b == src.size()) src.push_back(from[p]);
    owner[p] = b;
  }
  std::vector<cplx> G;
  if ((rc = greens_np(m, t, src, tgt, owner, broadening, precision, G))) return rc;
  const uint32_t E = t->E;
  const cplx i(0, 1);
  cplx *o = reinterpret_cast<cplx *>(out);
  for (uint32_t p = 0; p < P; p++) {
    // expectationValue -= weight*conj(i*G[e])*dE/M_PI
    cplx v = 0.;
    for (uint32_t e = 0; e < E; e++) v -= occupation[e] * std::conj(i * G[(size_t)p * E + e]) * dE / M_PI;
    o[p] = v;
  }
  return TBTKKPM_OK;
}
