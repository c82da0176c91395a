// Seeded synthetic sparse matrices and dense operands (host C++, OpenMP).
// Deterministic for a given seed regardless of thread count: every random
// draw comes from a counter-based hash of (seed, stream, index).
//
// They stand in for the datasets the reference evaluates on (SuiteSparse and
// graph .npz files, absent here), with the shapes and value distributions of
// the benchmark configurations:
//   uniform   : M x K, Poisson(mean) row lengths, columns uniform without
//               replacement, values U(-1, 1)
//   rmat      : R-MAT(a,b,c,d) 2^scale nodes, edge_factor*2^scale edges,
//               symmetrised, self-loops added, duplicates removed, values
//               D^-1/2 (A+I) D^-1/2 (GCN normalisation)
//   stencil27 : 27-point stencil on an n^3 grid, values N(0,1), diagonal
//               27 + |sum of the row's off-diagonal values|
//   zipf      : M x M, degrees Zipf(s) truncated to [dmin, dmax], columns
//               uniform without replacement, values U(0,1) row-normalised
//   banded / blockdiag : structured families for the schedule model
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <algorithm>
#include <numeric>
#include <vector>
#include <parallel/algorithm>
#include <omp.h>

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed * 0x100000001B3ull ^ stream) ^ i);
}
inline double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

struct Rng {  // sequential generator for one (seed, stream)
  uint64_t seed, stream, i = 0;
  Rng(uint64_t s, uint64_t st) : seed(s), stream(st) {}
  uint64_t next() { return hash3(seed, stream, i++); }
  double uniform() { return u01(next()); }
  double normal() {
    double a = uniform(), b = uniform();
    if (a < 1e-300) a = 1e-300;
    return sqrt(-2.0 * log(a)) * cos(6.283185307179586 * b);
  }
  int poisson(double mean) {  // inversion; fine for the small means used here
    double l = exp(-mean), p = 1.0;
    int k = 0;
    do { ++k; p *= uniform(); } while (p > l && k < 100000);
    return k - 1;
  }
};

struct Csr {
  int32_t M = 0, K = 0;
  std::vector<int32_t> rowptr, col;
  std::vector<float> val;
};

// Rows given as per-row column lists -> CSR (columns sorted per row).
void finish_rows(Csr& c, std::vector<std::vector<int32_t>>& rows) {
  c.rowptr.assign(c.M + 1, 0);
  for (int32_t i = 0; i < c.M; ++i) c.rowptr[i + 1] = c.rowptr[i] + (int32_t)rows[i].size();
  c.col.resize(c.rowptr[c.M]);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < c.M; ++i) {
    std::sort(rows[i].begin(), rows[i].end());
    std::copy(rows[i].begin(), rows[i].end(), c.col.begin() + c.rowptr[i]);
  }
}

void sample_distinct(Rng& r, int32_t K, int32_t k, std::vector<int32_t>& out) {
  out.clear();
  if (k >= K) {
    out.resize(K);
    std::iota(out.begin(), out.end(), 0);
    return;
  }
  if ((int64_t)k * 4 > K) {  // dense-ish: partial Fisher-Yates
    std::vector<int32_t> p(K);
    std::iota(p.begin(), p.end(), 0);
    for (int32_t i = 0; i < k; ++i) {
      int32_t j = i + (int32_t)(r.next() % (uint64_t)(K - i));
      std::swap(p[i], p[j]);
    }
    out.assign(p.begin(), p.begin() + k);
    return;
  }
  while ((int32_t)out.size() < k) {
    int32_t c = (int32_t)(r.next() % (uint64_t)K);
    if (std::find(out.begin(), out.end(), c) == out.end()) out.push_back(c);
  }
}

Csr* gen_uniform(int32_t M, int32_t K, double mean, uint64_t seed) {
  Csr* c = new Csr;
  c->M = M; c->K = K;
  std::vector<std::vector<int32_t>> rows(M);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < M; ++i) {
    Rng r(seed, 1000003ull * (uint64_t)i + 1);
    int k = r.poisson(mean);
    sample_distinct(r, K, k, rows[i]);
  }
  finish_rows(*c, rows);
  c->val.resize(c->col.size());
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)c->col.size(); ++e)
    c->val[e] = (float)(2.0 * u01(hash3(seed, 7, (uint64_t)e)) - 1.0);
  return c;
}

// Sorted unique (row << 32 | col) keys -> CSR.
void keys_to_csr(Csr& c, std::vector<uint64_t>& keys) {
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  c.rowptr.assign(c.M + 1, 0);
  c.col.resize(keys.size());
  for (size_t e = 0; e < keys.size(); ++e) c.rowptr[(keys[e] >> 32) + 1]++;
  for (int32_t i = 0; i < c.M; ++i) c.rowptr[i + 1] += c.rowptr[i];
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)keys.size(); ++e) c.col[e] = (int32_t)(keys[e] & 0xFFFFFFFFu);
}

void gcn_normalise(Csr& c) {
  c.val.resize(c.col.size());
  std::vector<double> isq(c.M);
  for (int32_t i = 0; i < c.M; ++i) {
    int32_t d = c.rowptr[i + 1] - c.rowptr[i];
    isq[i] = d > 0 ? 1.0 / sqrt((double)d) : 0.0;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t i = 0; i < c.M; ++i)
    for (int32_t e = c.rowptr[i]; e < c.rowptr[i + 1]; ++e)
      c.val[e] = (float)(isq[i] * isq[c.col[e]]);
}

Csr* gen_rmat(int32_t scale, double edge_factor, double a, double b, double cc, uint64_t seed) {
  Csr* c = new Csr;
  int32_t M = 1 << scale;
  c->M = M; c->K = M;
  int64_t E = (int64_t)(edge_factor * (double)M);
  std::vector<uint64_t> keys((size_t)(2 * E + M));
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < E; ++e) {
    uint64_t u = 0, v = 0;
    for (int l = 0; l < scale; ++l) {
      double x = u01(hash3(seed, 11 + l, (uint64_t)e));
      int q = x < a ? 0 : x < a + b ? 1 : x < a + b + cc ? 2 : 3;
      u = (u << 1) | (uint64_t)(q >> 1);
      v = (v << 1) | (uint64_t)(q & 1);
    }
    keys[2 * e] = (u << 32) | v;
    keys[2 * e + 1] = (v << 32) | u;
  }
  for (int32_t i = 0; i < M; ++i) keys[2 * E + i] = ((uint64_t)i << 32) | (uint64_t)i;
  keys_to_csr(*c, keys);
  gcn_normalise(*c);
  return c;
}

Csr* gen_stencil27(int32_t n, uint64_t seed) {
  Csr* c = new Csr;
  int64_t M64 = (int64_t)n * n * n;
  c->M = (int32_t)M64; c->K = c->M;
  c->rowptr.assign(c->M + 1, 0);
  auto count = [n](int64_t x) { return (x > 0) + 1 + (x < n - 1); };
  for (int64_t r = 0; r < M64; ++r) {
    int64_t z = r / ((int64_t)n * n), y = (r / n) % n, x = r % n;
    c->rowptr[r + 1] = c->rowptr[r] + (int32_t)(count(x) * count(y) * count(z));
  }
  c->col.resize(c->rowptr[c->M]);
  c->val.resize(c->col.size());
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < M64; ++r) {
    int64_t z = r / ((int64_t)n * n), y = (r / n) % n, x = r % n;
    int32_t e = c->rowptr[r];
    int32_t diag = -1;
    double sum = 0.0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int64_t zz = z + dz, yy = y + dy, xx = x + dx;
          if (zz < 0 || zz >= n || yy < 0 || yy >= n || xx < 0 || xx >= n) continue;
          c->col[e] = (int32_t)((zz * n + yy) * n + xx);
          Rng rr(seed, 5000011ull * (uint64_t)r + (uint64_t)(e - c->rowptr[r]));
          float v = (float)rr.normal();
          if (dz == 0 && dy == 0 && dx == 0) diag = e; else sum += v;
          c->val[e] = v;
          ++e;
        }
    c->val[diag] = (float)(27.0 + fabs(sum));
  }
  return c;
}

Csr* gen_zipf(int32_t M, double s, int32_t dmin, int32_t dmax, uint64_t seed) {
  Csr* c = new Csr;
  c->M = M; c->K = M;
  // inverse-CDF table of the truncated Zipf law on [dmin, dmax]
  std::vector<double> cdf(dmax - dmin + 1);
  double acc = 0.0;
  for (int d = dmin; d <= dmax; ++d) { acc += pow((double)d, -s); cdf[d - dmin] = acc; }
  for (auto& x : cdf) x /= acc;
  std::vector<std::vector<int32_t>> rows(M);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < M; ++i) {
    Rng r(seed, 7000003ull * (uint64_t)i + 3);
    double x = r.uniform();
    int d = dmin + (int)(std::lower_bound(cdf.begin(), cdf.end(), x) - cdf.begin());
    if (d > M) d = M;
    sample_distinct(r, M, d, rows[i]);
  }
  finish_rows(*c, rows);
  c->val.resize(c->col.size());
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < M; ++i) {
    double sum = 0.0;
    for (int32_t e = c->rowptr[i]; e < c->rowptr[i + 1]; ++e) {
      c->val[e] = (float)u01(hash3(seed, 9, (uint64_t)e));
      sum += c->val[e];
    }
    for (int32_t e = c->rowptr[i]; e < c->rowptr[i + 1]; ++e)
      c->val[e] = (float)(c->val[e] / (sum > 0 ? sum : 1.0));
  }
  return c;
}

// Banded: row i has columns within [i - bw, i + bw], each kept with prob. fill.
Csr* gen_banded(int32_t M, int32_t bw, double fill, uint64_t seed) {
  Csr* c = new Csr;
  c->M = M; c->K = M;
  std::vector<std::vector<int32_t>> rows(M);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < M; ++i) {
    Rng r(seed, 9000011ull * (uint64_t)i + 5);
    int32_t lo = i - bw < 0 ? 0 : i - bw, hi = i + bw >= M ? M - 1 : i + bw;
    for (int32_t j = lo; j <= hi; ++j)
      if (j == i || r.uniform() < fill) rows[i].push_back(j);
  }
  finish_rows(*c, rows);
  c->val.resize(c->col.size());
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)c->col.size(); ++e)
    c->val[e] = (float)(2.0 * u01(hash3(seed, 13, (uint64_t)e)) - 1.0);
  return c;
}

// Block-diagonal clusters of size bs with `deg` entries per row, a fraction
// `noise` of them placed uniformly off-block.
Csr* gen_blockdiag(int32_t M, int32_t bs, int32_t deg, double noise, uint64_t seed) {
  Csr* c = new Csr;
  c->M = M; c->K = M;
  std::vector<std::vector<int32_t>> rows(M);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < M; ++i) {
    Rng r(seed, 11000027ull * (uint64_t)i + 7);
    int32_t b0 = (i / bs) * bs, b1 = b0 + bs > M ? M : b0 + bs;
    std::vector<int32_t>& row = rows[i];
    int tries = 0;
    while ((int32_t)row.size() < deg && tries < 8 * deg) {
      ++tries;
      int32_t j = r.uniform() < noise ? (int32_t)(r.next() % (uint64_t)M)
                                      : b0 + (int32_t)(r.next() % (uint64_t)(b1 - b0));
      if (std::find(row.begin(), row.end(), j) == row.end()) row.push_back(j);
    }
  }
  finish_rows(*c, rows);
  c->val.resize(c->col.size());
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)c->col.size(); ++e)
    c->val[e] = (float)(2.0 * u01(hash3(seed, 17, (uint64_t)e)) - 1.0);
  return c;
}

}  // namespace

extern "C" {

void* dtcgen_uniform(int32_t M, int32_t K, double mean, uint64_t seed) {
  return gen_uniform(M, K, mean, seed);
}
void* dtcgen_rmat(int32_t scale, double edge_factor, double a, double b, double c,
                  uint64_t seed) {
  return gen_rmat(scale, edge_factor, a, b, c, seed);
}
void* dtcgen_stencil27(int32_t n, uint64_t seed) { return gen_stencil27(n, seed); }
void* dtcgen_zipf(int32_t M, double s, int32_t dmin, int32_t dmax, uint64_t seed) {
  return gen_zipf(M, s, dmin, dmax, seed);
}
void* dtcgen_banded(int32_t M, int32_t bw, double fill, uint64_t seed) {
  return gen_banded(M, bw, fill, seed);
}
void* dtcgen_blockdiag(int32_t M, int32_t bs, int32_t deg, double noise, uint64_t seed) {
  return gen_blockdiag(M, bs, deg, noise, seed);
}
void dtcgen_shape(void* h, int32_t* M, int32_t* K, int64_t* nnz) {
  Csr* c = (Csr*)h;
  *M = c->M; *K = c->K; *nnz = (int64_t)c->col.size();
}
void dtcgen_copy(void* h, int32_t* rowptr, int32_t* col, float* val) {
  Csr* c = (Csr*)h;
  memcpy(rowptr, c->rowptr.data(), (c->M + 1) * sizeof(int32_t));
  memcpy(col, c->col.data(), c->col.size() * sizeof(int32_t));
  if (val) memcpy(val, c->val.data(), c->val.size() * sizeof(float));
}
void dtcgen_free(void* h) { delete (Csr*)h; }

// Dense N(0,1) fill of n floats, element i from hash(seed, i).
void dtcgen_normal(float* out, int64_t n, uint64_t seed) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i += 2) {
    uint64_t h = hash3(seed, 3, (uint64_t)i);
    double a = u01(h), b = u01(mix64(h));
    if (a < 1e-300) a = 1e-300;
    double r = sqrt(-2.0 * log(a));
    out[i] = (float)(r * cos(6.283185307179586 * b));
    if (i + 1 < n) out[i + 1] = (float)(r * sin(6.283185307179586 * b));
  }
}

}  // extern "C"
