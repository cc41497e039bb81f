// Host-side pieces of the drop-in around the evaluation: the bias
// initialisation, the contact-map post-processing and the alignment / output
// file formats.  Each function keeps the reference's operation order in
// float, so results are bit-identical to the reference's C code on the same
// input (checked in tests/test_host.py against the compiled reference).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ccmpred_b200.h"

namespace {

constexpr int kQ = 21;
constexpr int kQPad = 32;

long long nsp_of(int L) {
  const long long ns = (long long)L * (kQ - 1);
  return ns + kQPad - ns % kQPad;
}

inline long long widx(int b, int k, int a, int j, int L) {
  return (((long long)b * L + k) * kQPad + a) * L + j;
}

// Alphabet of src/sequence.c:8-27: A R N D C Q E G H I L K M F P S T W Y V, gap/other = 20.
const unsigned char kAminoIndex[26] = {0,  20, 4,  3,  6,  13, 7,  8,  9,  20, 11, 10, 12,
                                       2,  20, 14, 5,  1,  15, 16, 20, 19, 17, 20, 18, 20};

unsigned char aa_to_index(unsigned char c) {
  if (!std::isalpha(c)) return 20;
  c = (unsigned char)std::toupper(c);
  if (c < 'A' || c > 'Z') return 20;
  return kAminoIndex[c - 'A'];
}

}  // namespace

namespace ccm {
void init_single_fields(const unsigned char *msa, int ncol, int nrow, float *x);
}

extern "C" {

// src/ccmpred.c:90-131: V(j,a) = log f_a - log f_gap from pseudocounted column
// frequencies, all couplings 0.
CCM_API void ccm_init_bias(const unsigned char *msa, int ncol, int nrow, float *x) {
  const long long nvar = ccm_nvar_padded(ncol);
  std::memset(x, 0, sizeof(float) * (size_t)nvar);
  ccm::init_single_fields(msa, ncol, nrow, x);
}

}  // extern "C"

namespace ccm {

// The single fields V of init_bias (src/ccmpred.c:101-129): x[a*L + j] for the
// 20 non-gap states; the rest of x is left as it is.
void init_single_fields(const unsigned char *msa, int ncol, int nrow, float *x) {
  for (int j = 0; j < ncol; ++j) {
    int counts[kQ];
    for (int a = 0; a < kQ; ++a) counts[a] = 1;
    for (int i = 0; i < nrow; ++i) counts[msa[(long long)i * ncol + j]]++;
    const int total = nrow + kQ;
    float frac[kQ];
    for (int a = 0; a < kQ; ++a) frac[a] = (float)counts[a] / total;
    const float gap_log = logf(frac[kQ - 1]);
    for (int a = 0; a < kQ - 1; ++a) x[(long long)a * ncol + j] = logf(frac[a]) - gap_log;
  }
}

}  // namespace ccm

extern "C" {

// src/util.c:16-64: Frobenius norm of the mean-centred 20x20 block of every
// column pair, zero diagonal.  Returns sqrt(sum of W^2 over k < j, 21x21).
CCM_API double ccm_sum_submatrices(const float *x, float *out, int ncol) {
  const float *x2 = x + nsp_of(ncol);
  std::memset(out, 0, sizeof(float) * (size_t)ncol * ncol);
  float xnorm = 0;
  for (int k = 0; k < ncol; ++k)
    for (int j = k + 1; j < ncol; ++j)
      for (int a = 0; a < kQ; ++a)
        for (int b = 0; b < kQ; ++b) {
          const float w = x2[widx(b, k, a, j, ncol)];
          xnorm += w * w;
        }
  for (int k = 0; k < ncol; ++k) {
    for (int j = 0; j < ncol; ++j) {
      float mean = 0;
      for (int a = 0; a < kQ; ++a)
        for (int b = 0; b < kQ; ++b) mean += x2[widx(b, k, a, j, ncol)];
      mean /= (kQ * kQ);
      for (int a = 0; a < kQ - 1; ++a)
        for (int b = 0; b < kQ - 1; ++b) {
          const float w = x2[widx(b, k, a, j, ncol)] - mean;
          out[(long long)k * ncol + j] += w * w;
        }
    }
  }
  for (int k = 0; k < ncol; ++k) {
    for (int j = 0; j < ncol; ++j) out[(long long)k * ncol + j] = sqrtf(out[(long long)k * ncol + j]);
    out[(long long)k * ncol + k] = 0.0f;
  }
  return std::sqrt((double)xnorm);
}

// src/util.c:66-108: average product correction, then shift so that the
// smallest off-diagonal entry is 0; zero diagonal.
CCM_API void ccm_apc(float *mat, int ncol) {
  std::vector<float> means(ncol, 0.0f);
  float meansum = 0;
  for (int i = 0; i < ncol; ++i)
    for (int j = 0; j < ncol; ++j) {
      const float w = mat[(long long)i * ncol + j];
      means[j] += w / ncol;
      meansum += w;
    }
  meansum /= ncol * ncol;
  for (int i = 0; i < ncol; ++i)
    for (int j = 0; j < ncol; ++j) mat[(long long)i * ncol + j] -= (means[i] * means[j]) / meansum;
  float minv = INFINITY;
  for (int i = 0; i < ncol; ++i)
    for (int j = i + 1; j < ncol; ++j)
      if (mat[(long long)i * ncol + j] < minv) minv = mat[(long long)i * ncol + j];
  for (int i = 0; i < ncol; ++i) {
    for (int j = 0; j < ncol; ++j) mat[(long long)i * ncol + j] -= minv;
    mat[(long long)i * ncol + i] = 0;
  }
}

// src/util.c:110-140: rescale off-diagonal entries to [0,1], zero diagonal.
// Returns CCM_ERR_INVALID when all off-diagonal entries are equal (the
// reference asserts).
CCM_API int ccm_normalize(float *mat, int ncol) {
  if (ncol < 2) return CCM_ERR_INVALID;
  float mn = mat[1], mx = mat[1];
  for (int i = 0; i < ncol; ++i)
    for (int j = 0; j < ncol; ++j) {
      if (i == j) continue;
      const float v = mat[(long long)i * ncol + j];
      if (v < mn) mn = v;
      if (v > mx) mx = v;
    }
  const float range = mx - mn;
  if (range == 0) return CCM_ERR_INVALID;
  for (int i = 0; i < ncol; ++i)
    for (int j = 0; j < ncol; ++j) {
      float v = mat[(long long)i * ncol + j];
      v = (v - mn) / range;
      mat[(long long)i * ncol + j] = (i == j) ? 0.0f : v;
    }
  return CCM_OK;
}

// src/io.c:20-28: "%.20e\t" per entry, newline per row.
CCM_API int ccm_write_matrix(const char *path, const float *mat, int ncol, int nrow) {
  FILE *f = std::fopen(path, "w");
  if (!f) return CCM_ERR_INVALID;
  for (int i = 0; i < nrow; ++i) {
    for (int j = 0; j < ncol; ++j) std::fprintf(f, "%.20e\t", mat[(long long)i * ncol + j]);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  return CCM_OK;
}

// src/io.c:31-60: L lines of the 20 single fields ("%g\t"), then for every
// pair i < j a "# i j" header and 21 lines of 21 couplings W(b,j,a,i) ("%.20e\t").
CCM_API int ccm_write_raw(const char *path, const float *x, int ncol) {
  FILE *f = std::fopen(path, "w");
  if (!f) return CCM_ERR_INVALID;
  const float *x2 = x + nsp_of(ncol);
  for (int i = 0; i < ncol; ++i) {
    for (int a = 0; a < kQ - 1; ++a) std::fprintf(f, "%g\t", x[(long long)a * ncol + i]);
    std::fprintf(f, "\n");
  }
  for (int i = 0; i < ncol; ++i)
    for (int j = i + 1; j < ncol; ++j) {
      std::fprintf(f, "# %d %d\n", i, j);
      for (int a = 0; a < kQ; ++a) {
        for (int b = 0; b < kQ; ++b) std::fprintf(f, "%.20e\t", x2[widx(b, j, a, i, ncol)]);
        std::fprintf(f, "\n");
      }
    }
  std::fclose(f);
  return CCM_OK;
}

// src/io.c:62-103: read a raw file written by ccm_write_raw / the reference
// into x (both symmetric halves of every coupling block).  x must hold
// nvar_padded floats and is not cleared first (as in the reference).
CCM_API int ccm_read_raw(const char *path, float *x, int ncol) {
  FILE *f = std::fopen(path, "r");
  if (!f) return CCM_ERR_INVALID;
  float *x2 = x + nsp_of(ncol);
  std::vector<char> line(1 << 16);
  int rc = CCM_OK;
  for (int i = 0; i < ncol && rc == CCM_OK; ++i) {
    if (!std::fgets(line.data(), (int)line.size(), f)) { rc = CCM_ERR_INVALID; break; }
    char *tok = line.data();
    for (int a = 0; a < kQ - 1; ++a) x[(long long)a * ncol + i] = (float)std::strtod(tok, &tok);
  }
  char expected[64];
  for (int i = 0; i < ncol && rc == CCM_OK; ++i)
    for (int j = i + 1; j < ncol && rc == CCM_OK; ++j) {
      if (!std::fgets(line.data(), (int)line.size(), f)) { rc = CCM_ERR_INVALID; break; }
      std::snprintf(expected, sizeof(expected), "# %d %d\n", i, j);
      if (std::strcmp(line.data(), expected) != 0) { rc = CCM_ERR_INVALID; break; }
      for (int a = 0; a < kQ; ++a) {
        if (!std::fgets(line.data(), (int)line.size(), f)) { rc = CCM_ERR_INVALID; break; }
        char *tok = line.data();
        for (int b = 0; b < kQ; ++b) {
          const float v = (float)std::strtod(tok, &tok);
          x2[widx(b, j, a, i, ncol)] = v;
          x2[widx(a, i, b, j, ncol)] = v;
        }
      }
    }
  std::fclose(f);
  return rc;
}

// src/sequence.c:48-80: PSICOV alignment, one sequence per line; rejects
// a3m/FASTA ('>'); ncol = longest trimmed line, shorter rows padded with gaps.
// Returns a malloc'd N x L array (free with ccm_free) or NULL.
CCM_API unsigned char *ccm_read_msa(const char *path, int *ncol, int *nrow) {
  FILE *f = std::fopen(path, "r");
  if (!f) return nullptr;
  std::vector<std::string> rows;
  std::vector<char> buf(1 << 16);
  int L = 0;
  while (std::fgets(buf.data(), (int)buf.size(), f)) {
    std::string s(buf.data());
    while (!s.empty() && std::isspace((unsigned char)s.back())) s.pop_back();
    if (s.find('>') != std::string::npos) {
      std::fclose(f);
      *ncol = *nrow = -1;
      return nullptr;
    }
    if ((int)s.size() > L) L = (int)s.size();
    rows.push_back(s);
  }
  std::fclose(f);
  const int N = (int)rows.size();
  unsigned char *out = static_cast<unsigned char *>(std::malloc((size_t)N * (L > 0 ? L : 1)));
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < L; ++j)
      out[(long long)i * L + j] = j < (int)rows[i].size() ? aa_to_index((unsigned char)rows[i][j]) : 20;
  *ncol = L;
  *nrow = N;
  return out;
}

CCM_API void ccm_free(void *p) { std::free(p); }

}  // extern "C"
