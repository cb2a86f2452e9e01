// exec_cpu.cpp — TEST-ONLY CPU executor for the library's planner.
//
// Binds curfp_b200/csrc/plan.cpp to plain loops (FP64 accumulation) so the
// -m "not gpu" tests can check view arithmetic, recursion splits, masks and
// info propagation of every RFP routine without a GPU.  It is compiled into
// tests/hostsim/libhostsim.so only; the product library never contains it.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <vector>

#include "engine.h"

using namespace rfp;

namespace {

inline float& at(View v, int64_t i, int64_t j) { return v.p[i * v.rs + j * v.cs]; }

class CpuExec : public Exec {
 public:
  int info = INT_MAX;
  bool abort_on_info = false;
  long gemm_calls = 0, inplace_calls = 0;
  std::vector<float> ws;

  bool aborted() const { return abort_on_info && info != INT_MAX; }

  int gemm(const GemmProb* p, int count) override {
    if (count > kMaxBatch) return 3;
    if (aborted()) return 0;
    ++gemm_calls;
    for (int t = 0; t < count; ++t) {
      const GemmProb& g = p[t];
      if (g.m <= 0 || g.n <= 0) continue;
      if (g.inplace) {
        ++inplace_calls;
        if (g.m > inplace_rows()) return 3;
      }
      std::vector<double> tmp((size_t)g.m * g.n, 0.0);
      for (int j = 0; j < g.n; ++j)
        for (int i = 0; i < g.m; ++i) {
          double s = 0.0;
          auto keep = [&](int at_, int bt_, int k) {
            return (at_ != 1 || k <= i) && (at_ != 2 || k >= i) && (at_ != 3 || k > i) &&
                   (bt_ != 1 || k >= j) && (bt_ != 2 || k <= j);
          };
          for (int k = 0; k < g.k; ++k)
            if (keep(g.a_tri, g.b_tri, k)) s += (double)at(g.A, i, k) * (double)at(g.B, k, j);
          for (int k = 0; k < g.k2; ++k)
            if (keep(g.a2_tri, g.b2_tri, k)) s += (double)at(g.A2, i, k) * (double)at(g.B2, k, j);
          tmp[(size_t)j * g.m + i] = s;
        }
      for (int j = 0; j < g.n; ++j)
        for (int i = 0; i < g.m; ++i) {
          if (g.c_lower && j > i) continue;
          double v = g.alpha * tmp[(size_t)j * g.m + i];
          if (g.beta != 0.0f) v += (double)g.beta * at(g.C, i, j);
          at(g.C, i, j) = (float)v;
        }
    }
    return 0;
  }

  int potrf_tile(View L, int n, int info_base) override {
    if (info != INT_MAX) return 0;
    if (n > kPotrfTile) return 3;
    for (int j = 0; j < n; ++j) {
      double d = at(L, j, j);
      if (!(d > 0.0)) {
        if (info_base + j + 1 < info) info = info_base + j + 1;
        return 0;
      }
      d = std::sqrt(d);
      at(L, j, j) = (float)d;
      for (int i = j + 1; i < n; ++i) at(L, i, j) = (float)(at(L, i, j) / d);
      for (int k = j + 1; k < n; ++k)
        for (int i = k; i < n; ++i)
          at(L, i, k) = (float)((double)at(L, i, k) - (double)at(L, i, j) * at(L, k, j));
    }
    return 0;
  }

  static void inv_lower(View L, int r0, int sz, std::vector<double>& X) {
    X.assign((size_t)sz * sz, 0.0);
    for (int c = 0; c < sz; ++c)
      for (int i = c; i < sz; ++i) {
        double s = (i == c) ? 1.0 : 0.0;
        for (int k = c; k < i; ++k) s -= (double)at(L, r0 + i, r0 + k) * X[(size_t)k * sz + c];
        X[(size_t)i * sz + c] = s / at(L, r0 + i, r0 + i);
      }
  }

  int trtri_blocks(View L, int n, int nb, float* W) override {
    if (aborted()) return 0;
    std::vector<double> X;
    for (int b = 0; b * nb < n; ++b) {
      int r0 = b * nb, sz = std::min(nb, n - r0);
      inv_lower(L, r0, sz, X);
      float* Wb = W + (int64_t)b * kInvStride;
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i)
          Wb[(int64_t)j * nb + i] = (i < sz && j < sz && i >= j) ? (float)X[(size_t)i * sz + j] : 0.f;
    }
    return 0;
  }

  int trtri_tile(View L, int n) override {
    if (n > kTriTile) return 3;
    std::vector<double> X;
    inv_lower(L, 0, n, X);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j <= i; ++j) at(L, i, j) = (float)X[(size_t)i * n + j];
    return 0;
  }

  int lauum_tile(View L, int n) override {
    if (n > kTriTile) return 3;
    std::vector<double> R((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = 0.0;
        for (int k = i; k < n; ++k) s += (double)at(L, k, i) * at(L, k, j);
        R[(size_t)i * n + j] = s;
      }
    for (int i = 0; i < n; ++i)
      for (int j = 0; j <= i; ++j) at(L, i, j) = (float)R[(size_t)i * n + j];
    return 0;
  }

  // Same block algorithm as the GPU wavefront kernel: X_j = W_j (alpha B_j -
  // sum_{i<j} L_ji X_i), blocks of 64.
  long wave_calls = 0;
  int trsm_wave(View L, int n, View B, int m, float alpha, const float* W) override {
    if (aborted()) return 0;
    ++wave_calls;
    const int NB = kTrsmLeaf;
    std::vector<double> T((size_t)NB * m);
    for (int r0 = 0; r0 < n; r0 += NB) {
      const int rows = std::min(NB, n - r0), j = r0 / NB;
      for (int a = 0; a < rows; ++a)
        for (int c = 0; c < m; ++c) {
          double s = (double)alpha * at(B, r0 + a, c);
          for (int k = 0; k < r0; ++k) s -= (double)at(L, r0 + a, k) * at(B, k, c);
          T[(size_t)a * m + c] = s;
        }
      const float* Wj = W + (int64_t)j * kInvStride;
      for (int a = 0; a < rows; ++a)
        for (int c = 0; c < m; ++c) {
          double s = 0;
          for (int k = 0; k < rows; ++k) s += (double)Wj[(int64_t)k * NB + a] * T[(size_t)k * m + c];
          at(B, r0 + a, c) = (float)s;
        }
    }
    return 0;
  }

  // Same column recurrence as the GPU tile kernel, in FP64.
  int potrf_adj_tile(View L, View G, int n) override {
    if (n > kAdjTile) return 3;
    std::vector<double> l((size_t)n * n, 0.0), g((size_t)n * n, 0.0);
    for (int p = 0; p < n; ++p)
      for (int q = 0; q <= p; ++q) {
        l[(size_t)p * n + q] = at(L, p, q);
        g[(size_t)p * n + q] = at(G, p, q);
      }
    for (int j = n - 1; j >= 0; --j) {
      const double lj = l[(size_t)j * n + j];
      for (int p = j + 1; p < n; ++p) {
        double w = 0.0;
        for (int q = j + 1; q < n; ++q) {
          const double gv = q < p ? g[(size_t)p * n + q]
                                  : (q > p ? g[(size_t)q * n + p] : 2.0 * g[(size_t)p * n + p]);
          w += gv * l[(size_t)q * n + j];
        }
        g[(size_t)p * n + j] = (g[(size_t)p * n + j] - w) / lj;
      }
      double d = 0.0;
      for (int p = j + 1; p < n; ++p) d += g[(size_t)p * n + j] * l[(size_t)p * n + j];
      g[(size_t)j * n + j] = (g[(size_t)j * n + j] - d) / (2.0 * lj);
    }
    for (int p = 0; p < n; ++p)
      for (int q = 0; q <= p; ++q) at(G, p, q) = (float)g[(size_t)p * n + q];
    return 0;
  }

  float* workspace(size_t nfloats) override {
    if (ws.size() < nfloats) ws.resize(nfloats);
    return ws.data();
  }
  int inplace_rows() const override { return 64; }
};

}  // namespace

extern "C" {

int hs_ssfrk(int transr, int lower, int trans, int n, int k, float alpha,
             const float* A, int lda, float beta, float* C, long* calls) {
  CpuExec ex;
  int rc = plan::ssfrk(ex, transr, lower, trans, n, k, alpha, A, lda, beta, C);
  if (calls) *calls = ex.gemm_calls;
  return rc;
}

int hs_ssfr2k(int transr, int lower, int trans, int n, int k, float alpha,
              const float* A, int lda, const float* B, int ldb, float beta, float* C) {
  CpuExec ex;
  return plan::ssfr2k(ex, transr, lower, trans, n, k, alpha, A, lda, B, ldb, beta, C);
}

int hs_spftrf(int transr, int lower, int n, float* A, int* info) {
  CpuExec ex;
  ex.abort_on_info = true;
  int rc = plan::spftrf(ex, transr, lower, n, A);
  *info = ex.info == INT_MAX ? 0 : ex.info;
  return rc;
}

int hs_spftrs(int transr, int lower, int n, int nrhs, const float* A, float* B, int ldb) {
  CpuExec ex;
  return plan::spftrs(ex, transr, lower, n, nrhs, A, B, ldb);
}

int hs_spftri(int transr, int lower, int n, float* A) {
  CpuExec ex;
  return plan::spftri(ex, transr, lower, n, A);
}

// Cholesky adjoint in RFP (same planning as curfpSpftrfBackward): G holds
// the factor's cotangent on entry and the matrix's on exit (RFP, in place).
int hs_spftrf_backward(int transr, int lower, int n, const float* L, float* G, int math,
                       long* calls) {
  CpuExec ex;
  int rc = plan::spftrf_adjoint(ex, transr, lower, n, L, G, math);
  if (calls) *calls = ex.gemm_calls;
  return rc;
}

// Same arithmetic as curfpSsfrkBackward.
int hs_ssfrk_backward(int transr, int lower, int trans, int n, int k, float alpha,
                      const float* A, int lda, const float* Cbar, float* Abar, int ldabar) {
  CpuExec ex;
  View X = trans ? View{const_cast<float*>(A), lda, 1} : View{const_cast<float*>(A), 1, lda};
  View Y = trans ? View{Abar, ldabar, 1} : View{Abar, 1, ldabar};
  return plan::rfp_symm_dbl(ex, transr, lower, n, Cbar, X, Y, k, alpha, 0.0f);
}

// Same sequence as curfpSpftrsBackward (column-major n x nrhs blocks, ld n).
int hs_spftrs_backward(int transr, int lower, int n, int nrhs, const float* L, const float* X,
                       const float* Xbar, float* Bbar, float* Lbar) {
  CpuExec ex;
  for (size_t e = 0; e < (size_t)n * nrhs; ++e) Bbar[e] = Xbar[e];
  int rc = plan::spftrs(ex, transr, lower, n, nrhs, L, Bbar, n);
  if (rc) return rc;
  std::vector<float> W((size_t)2 * n * nrhs);
  for (size_t e = 0; e < (size_t)n * nrhs; ++e) {
    W[e] = X[e];
    W[(size_t)n * nrhs + e] = Bbar[e];
  }
  View Wv{W.data(), 1, n};
  if ((rc = plan::rfp_trmm_t(ex, transr, lower, n, L, Wv, 2 * nrhs))) return rc;
  return plan::rfp_gemm_lower2(ex, transr, lower, n, Lbar, View{Bbar, 1, n}, tr(Wv),
                               View{const_cast<float*>(X), 1, n},
                               tr(View{W.data() + (size_t)n * nrhs, 1, n}), nrhs, -1.0f, 0.0f);
}

// rfp_trsm: L X = alpha B (trans 0) or L^T X = alpha B (trans 1); B column-major ld n.
int hs_rfp_trsm(int transr, int lower, int n, const float* L, int trans, float* B, int m,
                float alpha) {
  CpuExec ex;
  return plan::rfp_trsm(ex, transr, lower, n, L, trans, View{B, 1, n}, m, alpha, 0);
}

// Same planning as curfpSsfmm (side 0 left, 1 right; B, C column-major m x n).
int hs_ssfmm(int transr, int lower, int side, int m, int n, float alpha, const float* A,
             const float* B, int ldb, float beta, float* C, int ldc) {
  CpuExec ex;
  View Bv{const_cast<float*>(B), 1, ldb}, Cv{C, 1, ldc};
  if (side) {
    Bv = tr(Bv);
    Cv = tr(Cv);
  }
  return plan::rfp_symm(ex, transr, lower, side ? n : m, A, Bv, Cv, side ? m : n, alpha, beta);
}

int hs_geometry(int n, int transr, int lower, int64_t* out) {
  Geometry g = geometry(n, transr, lower);
  int64_t v[11] = {g.n1, g.n2, g.b11.off, g.b11.rs, g.b11.cs, g.b21.off, g.b21.rs,
                   g.b21.cs, g.b22.off, g.b22.rs, g.b22.cs};
  for (int i = 0; i < 11; ++i) out[i] = v[i];
  return 0;
}

}  // extern "C"
