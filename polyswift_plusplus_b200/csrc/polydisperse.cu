// polyDisperseBCP (pspolymer/PsPolyDisperseBCP.cpp:41-455) as quadrature chains,
// and the generalized Gauss-Laguerre rule it integrates the Schulz distribution with.
//
// The rule comes from the eigen-decomposition of the symmetric tridiagonal
// Jacobi matrix of the monic generalized Laguerre polynomials (Golub & Welsch,
// Math. Comp. 23 (1969) 221-230): diagonal 2i + a + 1, off-diagonal
// sqrt(i (i + a)); nodes are its eigenvalues, weights Gamma(a + 1) times the
// squared first components of its normalised eigenvectors.  The eigenproblem
// is solved by cyclic Jacobi rotations (n <= 64, so a dense solver is cheap
// and accurate to a few ulps).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "engine_state.h"

namespace psb {

static int gauss_laguerre_rule(int n, double a, double* x, double* w) {
  if (n < 1 || n > 64 || !(a > -1.0)) return PS_ATTRIB_ERR;
  std::vector<double> A((size_t)n * n, 0.0), V((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    A[(size_t)i * n + i] = 2.0 * i + a + 1.0;
    V[(size_t)i * n + i] = 1.0;
    if (i > 0) {
      const double e = sqrt((double)i * ((double)i + a));
      A[(size_t)i * n + i - 1] = e;
      A[(size_t)(i - 1) * n + i] = e;
    }
  }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int p = 0; p < n; ++p) {
      diag += A[(size_t)p * n + p] * A[(size_t)p * n + p];
      for (int q = p + 1; q < n; ++q) off += A[(size_t)p * n + q] * A[(size_t)p * n + q];
    }
    if (off <= 1e-34 * diag) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; ++k) {  // A <- A G (columns p, q)
          const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = c * akp - s * akq;
          A[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // A <- G^T A (rows p, q)
          const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = c * apk - s * aqk;
          A[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {  // V <- V G
          const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = c * vkp - s * vkq;
          V[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  const double mu0 = tgamma(a + 1.0);
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::sort(order.begin(), order.end(),
            [&](int i, int j) { return A[(size_t)i * n + i] < A[(size_t)j * n + j]; });
  for (int r = 0; r < n; ++r) {
    const int i = order[r];
    x[r] = A[(size_t)i * n + i];
    w[r] = mu0 * V[(size_t)i] * V[(size_t)i];  // first component of eigenvector i
  }
  return PS_OK;
}

int expand_polydisperse(ps_handle* h, const ps_config& in, ps_config* out) {
  *out = in;
  if (in.n_polymers < 1 || in.n_polymers > PS_MAX_POLYMERS) {
    h->err = "n_polymers out of range";
    return PS_ATTRIB_ERR;
  }
  h->chain_user.clear(); h->chain_k.clear(); h->chain_dwt.clear(); h->chain_vf.clear();
  h->user_first.clear(); h->user_ng.clear();
  int nc = 0;
  for (int ip = 0; ip < in.n_polymers; ++ip) {
    const ps_polymer_config& P = in.polymers[ip];
    const ps_polydisperse_config& D = in.polydisperse[ip];
    h->user_first.push_back(nc);
    if (!D.enabled) {
      if (nc >= PS_MAX_POLYMERS) {
        h->err = "too many polymers after the polydisperse expansion";
        return PS_ATTRIB_ERR;
      }
      out->polymers[nc] = P;
      memcpy(out->block_charge[nc], in.block_charge[ip], sizeof(in.block_charge[ip]));
      out->polydisperse[nc].enabled = 0;
      h->chain_user.push_back(ip); h->chain_k.push_back(0);
      h->chain_dwt.push_back(1.0); h->chain_vf.push_back(P.volfrac);
      h->user_ng.push_back(1);
      ++nc;
      continue;
    }
    // PsPolyDisperseBCP::setAttrib / calcPolyParams (pspolymer/PsPolyDisperseBCP.cpp:41-145, 384-455)
    if (P.n_blocks < 1 || P.n_blocks > 2) {
      h->err = "polyDisperseBCP: polydisperse model with more than two blocks not yet supported";
      return PS_ATTRIB_ERR;
    }
    if (D.poly_block < 0 || D.poly_block >= P.n_blocks || D.n_g < 1 || !(D.alpha > 0.0)) {
      h->err = "polyDisperseBCP: polyblock, n_g or alpha out of range";
      return PS_ATTRIB_ERR;
    }
    if (nc + D.n_g > PS_MAX_POLYMERS) {
      h->err = "too many polymers after the polydisperse expansion (n_g too large)";
      return PS_ATTRIB_ERR;
    }
    std::vector<double> x(D.n_g), w(D.n_g);
    int rc = gauss_laguerre_rule(D.n_g, D.alpha - 1.0, x.data(), w.data());
    if (rc) {
      h->err = "polyDisperseBCP: Gauss-Laguerre rule failed";
      return rc;
    }
    const double galpha = tgamma(D.alpha);
    const double nlen = (double)P.length;
    const double poly_frac = P.blocks[D.poly_block].lengthfrac;
    const double const_frac = 1.0 - poly_frac;
    const double nc_len = const_frac * nlen;
    const double n_b = (nlen - nc_len) / D.alpha;
    for (int k = 0; k < D.n_g; ++k) {
      ps_polymer_config C = P;
      C.blocks[D.poly_block].lengthfrac = ((x[k] * n_b + nc_len) / nlen) - const_frac;
      out->polymers[nc] = C;
      memcpy(out->block_charge[nc], in.block_charge[ip], sizeof(in.block_charge[ip]));
      out->polydisperse[nc] = D;
      h->chain_user.push_back(ip); h->chain_k.push_back(k);
      h->chain_dwt.push_back(w[k] / galpha); h->chain_vf.push_back(P.volfrac);
      ++nc;
    }
    h->user_ng.push_back(D.n_g);
  }
  out->n_polymers = nc;
  return PS_OK;
}

}  // namespace psb

extern "C" int ps_gauss_laguerre(int n, double a, double* x, double* w) {
  if (!x || !w) return PS_ATTRIB_ERR;
  return psb::gauss_laguerre_rule(n, a, x, w);
}
