/*
 * ORACLE — test infrastructure only. Never linked into the product library.
 *
 * Plain-C restatement of the haploid Li-Stephens imputation HMM of
 * GLIMPSE2_phase, in double precision (the FP64 reference for precision
 * reporting) and in single precision with sequential sums (checked against the
 * reference's own compiled code within 1e-5):
 *   - conditioning set: polymorphic sites and Hvar bits
 *     (phase/src/containers/conditioning_set.cpp:123-182),
 *   - transitions (conditioning_set.cpp:184-196),
 *   - emissions (phase/src/models/imputation_hmm.cpp:124-134),
 *   - forward pass with per-site rescaling (imputation_hmm.cpp:143-235),
 *   - backward pass and posteriors (imputation_hmm.cpp:237-416),
 *   - monomorphic sites (imputation_hmm.cpp:417-429).
 * rs_impute also returns the chunk log-likelihood sum_l log(AlphaSum_l) of the
 * forward rescaling (no counterpart in the reference).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define DEFINE_IMPUTE(NAME, REAL)                                                                                 \
  static double NAME(int L, const uint8_t* common, const uint8_t* lq, const uint8_t* major, const double* cm,      \
                     const int32_t* comrow, const uint8_t* hvar, int stride, const int64_t* shap_off,            \
                     const int32_t* shap_sites, const uint32_t* states, int K, double nrho, float ed_f, float ee_f,  \
                     const float* HL, const uint8_t* flat, float* HP) {                                          \
    const REAL ed = (REAL)ed_f, ee = (REAL)ee_f;                                                                  \
    uint8_t* poly = (uint8_t*)calloc(L, 1);                                                                       \
    int32_t* plist = (int32_t*)malloc(sizeof(int32_t) * L);                                                       \
    int np = 0;                                                                                                   \
    for (int l = 0; l < L; ++l) poly[l] = common[l];                                                              \
    for (int k = 0; k < K; ++k)                                                                                   \
      for (int64_t j = shap_off[states[k]]; j < shap_off[states[k] + 1]; ++j) poly[shap_sites[j]] = 1;            \
    for (int l = 0; l < L; ++l)                                                                                   \
      if (poly[l]) plist[np++] = l;                                                                               \
    uint8_t* bits = (uint8_t*)malloc((size_t)np * K + 1);                                                         \
    int32_t* lrel = (int32_t*)malloc(sizeof(int32_t) * L);                                                        \
    for (int i = 0; i < np; ++i) lrel[plist[i]] = i;                                                              \
    for (int i = 0; i < np; ++i) {                                                                                \
      const int s = plist[i];                                                                                     \
      for (int k = 0; k < K; ++k) {                                                                               \
        if (common[s]) {                                                                                          \
          const int h = (int)states[k];                                                                           \
          bits[(size_t)i * K + k] = (hvar[(size_t)comrow[s] * stride + (h >> 3)] >> (7 - (h & 7))) & 1;           \
        } else {                                                                                                  \
          bits[(size_t)i * K + k] = major[s];                                                                     \
        }                                                                                                         \
      }                                                                                                           \
    }                                                                                                             \
    for (int k = 0; k < K; ++k)                                                                                   \
      for (int64_t j = shap_off[states[k]]; j < shap_off[states[k] + 1]; ++j) {                                   \
        const int s = shap_sites[j];                                                                              \
        bits[(size_t)lrel[s] * K + k] = !major[s];                                                                \
      }                                                                                                           \
    REAL* t = (REAL*)malloc(sizeof(REAL) * (np + 1));                                                             \
    for (int i = 1; i < np; ++i) {                                                                                \
      double x = -expm1(nrho * (cm[plist[i]] - cm[plist[i - 1]]));                                                \
      x = x < 1e-7 ? 1e-7 : (x > 1.0 - 1e-7 ? 1.0 - 1e-7 : x);                                                    \
      t[i - 1] = (REAL)(float)x;                                                                                  \
    }                                                                                                             \
    REAL* alpha = (REAL*)malloc(sizeof(REAL) * (size_t)np * K + 1);                                               \
    REAL* asum = (REAL*)malloc(sizeof(REAL) * (np + 1));                                                          \
    REAL* beta = (REAL*)malloc(sizeof(REAL) * (K + 1));                                                           \
    double loglik = 0.0;                                                                                          \
    for (int i = 0; i < np; ++i) {                                                                                \
      const int s = plist[i];                                                                                     \
      const int fl = flat[s] || lq[s];                                                                            \
      REAL e[2];                                                                                                  \
      {                                                                                                           \
        const REAL p0 = (REAL)HL[2 * s] * ee + (REAL)HL[2 * s + 1] * ed;                                          \
        const REAL p1 = (REAL)HL[2 * s] * ed + (REAL)HL[2 * s + 1] * ee;                                          \
        e[0] = p0 / (p0 + p1);                                                                                    \
        e[1] = p1 / (p0 + p1);                                                                                    \
      }                                                                                                           \
      REAL sum = 0;                                                                                               \
      REAL* a = alpha + (size_t)i * K;                                                                            \
      if (i == 0) {                                                                                               \
        for (int k = 0; k < K; ++k) {                                                                             \
          a[k] = fl ? (REAL)1 / (REAL)K : e[bits[k]] * ((REAL)1 / (REAL)K);                                        \
          sum += a[k];                                                                                            \
        }                                                                                                         \
        if (fl) sum = 1;                                                                                          \
      } else {                                                                                                    \
        const REAL f1 = t[i - 1] / (REAL)K, f2 = ((REAL)1 - t[i - 1]) / asum[i - 1];                              \
        const REAL* ap = alpha + (size_t)(i - 1) * K;                                                             \
        for (int k = 0; k < K; ++k) {                                                                             \
          a[k] = ap[k] * f2 + f1;                                                                                 \
          if (!fl) a[k] *= e[bits[(size_t)i * K + k]];                                                            \
          sum += a[k];                                                                                            \
        }                                                                                                         \
      }                                                                                                           \
      asum[i] = sum;                                                                                              \
      loglik += log((double)sum);                                                                                 \
    }                                                                                                             \
    REAL bsum_next = 0;                                                                                           \
    for (int i = np - 1; i >= 0; --i) {                                                                           \
      const int s = plist[i];                                                                                     \
      const int fl = flat[s] || lq[s];                                                                            \
      REAL e[2];                                                                                                  \
      {                                                                                                           \
        const REAL p0 = (REAL)HL[2 * s] * ee + (REAL)HL[2 * s + 1] * ed;                                          \
        const REAL p1 = (REAL)HL[2 * s] * ed + (REAL)HL[2 * s + 1] * ee;                                          \
        e[0] = p0 / (p0 + p1);                                                                                    \
        e[1] = p1 / (p0 + p1);                                                                                    \
      }                                                                                                           \
      REAL ph[2] = {0, 0}, bsum = 0;                                                                              \
      const REAL* a = alpha + (size_t)i * K;                                                                      \
      const uint8_t* bi = bits + (size_t)i * K;                                                                   \
      if (i == np - 1) {                                                                                          \
        for (int k = 0; k < K; ++k) {                                                                             \
          ph[bi[k]] += a[k];                                                                                      \
          beta[k] = fl ? (REAL)1 / (REAL)K : e[bi[k]] * ((REAL)1 / (REAL)K);                                        \
          bsum += beta[k];                                                                                        \
        }                                                                                                         \
        if (fl) bsum = 1;                                                                                         \
      } else {                                                                                                    \
        const REAL f1 = t[i] / (REAL)K, f2 = ((REAL)1 - t[i]) / bsum_next;                                        \
        for (int k = 0; k < K; ++k) {                                                                             \
          const REAL pc = beta[k] * f2 + f1;                                                                      \
          ph[bi[k]] += a[k] * pc;                                                                                 \
          beta[k] = fl ? pc : pc * e[bi[k]];                                                                      \
          bsum += beta[k];                                                                                        \
        }                                                                                                         \
      }                                                                                                           \
      REAL po0, po1;                                                                                              \
      if (fl) {                                                                                                   \
        po0 = ph[0] * ee + ph[1] * ed;                                                                            \
        po1 = ph[0] * ed + ph[1] * ee;                                                                            \
        if (!flat[s]) {                                                                                           \
          po0 *= (REAL)HL[2 * s];                                                                                 \
          po1 *= (REAL)HL[2 * s + 1];                                                                             \
        }                                                                                                         \
      } else {                                                                                                    \
        const REAL h0 = ph[0] / e[0], h1 = ph[1] / e[1];                                                          \
        po0 = (h0 * ee + h1 * ed) * (REAL)HL[2 * s];                                                              \
        po1 = (h0 * ed + h1 * ee) * (REAL)HL[2 * s + 1];                                                          \
      }                                                                                                           \
      HP[2 * s] = (float)(po0 / (po0 + po1));                                                                     \
      HP[2 * s + 1] = (float)(po1 / (po0 + po1));                                                                 \
      bsum_next = bsum;                                                                                           \
    }                                                                                                             \
    for (int l = 0; l < L; ++l) {                                                                                 \
      if (poly[l]) continue;                                                                                      \
      REAL p0 = major[l] ? ed : ee, p1 = major[l] ? ee : ed;                                                      \
      if (!flat[l]) {                                                                                             \
        p0 *= (REAL)HL[2 * l];                                                                                    \
        p1 *= (REAL)HL[2 * l + 1];                                                                                \
      }                                                                                                           \
      HP[2 * l] = (float)(p0 / (p0 + p1));                                                                        \
      HP[2 * l + 1] = (float)(p1 / (p0 + p1));                                                                    \
    }                                                                                                             \
    free(poly); free(plist); free(bits); free(lrel); free(t); free(alpha); free(asum); free(beta);                \
    return loglik;                                                                                                \
  }

DEFINE_IMPUTE(impute_f64, double)
DEFINE_IMPUTE(impute_f32, float)

/* HP for one haplotype with conditioning set `states` (sorted reference ids).
 * precision: 64 or 32. Returns the chunk log-likelihood. */
double rs_impute(int precision, int L, const uint8_t* common, const uint8_t* lq, const uint8_t* major,
                 const double* cm, const int32_t* comrow, const uint8_t* hvar, int stride, const int64_t* shap_off,
                 const int32_t* shap_sites, const uint32_t* states, int K, double nrho, float ed, float ee,
                 const float* HL, const uint8_t* flat, float* HP) {
  if (precision == 64)
    return impute_f64(L, common, lq, major, cm, comrow, hvar, stride, shap_off, shap_sites, states, K, nrho, ed, ee,
                      HL, flat, HP);
  return impute_f32(L, common, lq, major, cm, comrow, hvar, stride, shap_off, shap_sites, states, K, nrho, ed, ee, HL,
                    flat, HP);
}

/* Per-window state posteriors, FP64: the label HMM of the learned state
 * selection (no counterpart in the reference). For the conditioning set built
 * as above, mass[w * K + k] = sum over the polymorphic sites l with
 * site_win[l] == w of alpha_l(k) beta_l(k) / sum_k' alpha_l(k') beta_l(k'),
 * alpha_l including the emission at l and beta_l the backward message
 * without it (beta = 1 at the last site); nsites[w] counts those sites. */
void rs_state_post(int L, const uint8_t* common, const uint8_t* lq, const uint8_t* major, const double* cm,
                   const int32_t* comrow, const uint8_t* hvar, int stride, const int64_t* shap_off,
                   const int32_t* shap_sites, const uint32_t* states, int K, double nrho, float ed_f, float ee_f,
                   const float* HL, const uint8_t* flat, const int32_t* site_win, int nwin, double* mass,
                   int32_t* nsites) {
  const double ed = ed_f, ee = ee_f;
  uint8_t* poly = (uint8_t*)calloc(L, 1);
  int32_t* plist = (int32_t*)malloc(sizeof(int32_t) * L);
  int np = 0;
  for (int l = 0; l < L; ++l) poly[l] = common[l];
  for (int k = 0; k < K; ++k)
    for (int64_t j = shap_off[states[k]]; j < shap_off[states[k] + 1]; ++j) poly[shap_sites[j]] = 1;
  for (int l = 0; l < L; ++l)
    if (poly[l]) plist[np++] = l;
  uint8_t* bits = (uint8_t*)malloc((size_t)np * K + 1);
  int32_t* lrel = (int32_t*)malloc(sizeof(int32_t) * L);
  for (int i = 0; i < np; ++i) lrel[plist[i]] = i;
  for (int i = 0; i < np; ++i) {
    const int s = plist[i];
    for (int k = 0; k < K; ++k) {
      const int h = (int)states[k];
      bits[(size_t)i * K + k] =
          common[s] ? (hvar[(size_t)comrow[s] * stride + (h >> 3)] >> (7 - (h & 7))) & 1 : major[s];
    }
  }
  for (int k = 0; k < K; ++k)
    for (int64_t j = shap_off[states[k]]; j < shap_off[states[k] + 1]; ++j)
      bits[(size_t)lrel[shap_sites[j]] * K + k] = !major[shap_sites[j]];
  double* t = (double*)malloc(sizeof(double) * (np + 1));
  for (int i = 1; i < np; ++i) {
    double x = -expm1(nrho * (cm[plist[i]] - cm[plist[i - 1]]));
    x = x < 1e-7 ? 1e-7 : (x > 1.0 - 1e-7 ? 1.0 - 1e-7 : x);
    t[i - 1] = (double)(float)x;
  }
  double* alpha = (double*)malloc(sizeof(double) * (size_t)np * K + 8);
  double* beta = (double*)malloc(sizeof(double) * (K + 1));
  double* nb = (double*)malloc(sizeof(double) * (K + 1));
  double* em = (double*)malloc(sizeof(double) * 2 * (np + 1));
  for (int i = 0; i < np; ++i) {
    const int s = plist[i];
    if (flat[s] || lq[s]) {
      em[2 * i] = em[2 * i + 1] = 1.0;
    } else {
      const double p0 = (double)HL[2 * s] * ee + (double)HL[2 * s + 1] * ed;
      const double p1 = (double)HL[2 * s] * ed + (double)HL[2 * s + 1] * ee;
      em[2 * i] = p0 / (p0 + p1);
      em[2 * i + 1] = p1 / (p0 + p1);
    }
  }
  for (int i = 0; i < np; ++i) {
    double* a = alpha + (size_t)i * K;
    double sum = 0;
    for (int k = 0; k < K; ++k) {
      const double prev = i == 0 ? 1.0 / K : alpha[(size_t)(i - 1) * K + k] * (1.0 - t[i - 1]) + t[i - 1] / K;
      a[k] = prev * em[2 * i + bits[(size_t)i * K + k]];
      sum += a[k];
    }
    for (int k = 0; k < K; ++k) a[k] /= sum;
  }
  for (int w = 0; w < nwin; ++w) nsites[w] = 0;
  for (size_t j = 0; j < (size_t)nwin * K; ++j) mass[j] = 0.0;
  for (int k = 0; k < K; ++k) beta[k] = 1.0;
  for (int i = np - 1; i >= 0; --i) {
    if (i < np - 1) {
      double se = 0;
      for (int k = 0; k < K; ++k) {
        nb[k] = em[2 * (i + 1) + bits[(size_t)(i + 1) * K + k]] * beta[k];
        se += nb[k];
      }
      for (int k = 0; k < K; ++k) beta[k] = nb[k] / se * (1.0 - t[i]) + t[i] / K;
    }
    const double* a = alpha + (size_t)i * K;
    double z = 0;
    for (int k = 0; k < K; ++k) z += a[k] * beta[k];
    const int w = site_win[plist[i]];
    nsites[w]++;
    for (int k = 0; k < K; ++k) mass[(size_t)w * K + k] += a[k] * beta[k] / z;
  }
  free(poly); free(plist); free(bits); free(lrel); free(t); free(alpha); free(beta); free(nb); free(em);
}
