// EMC FP64 oracle -- TEST INFRASTRUCTURE ONLY (see emc_oracle.h for the
// parity anchors).  Built with -ffp-contract=off so the FP32 voxel-index
// arithmetic below rounds exactly like the CUDA kernels, which use the same
// explicit fmaf/mul/add sequence.
#include "emc_oracle.h"

#include <algorithm>
#include <array>
#include <initializer_list>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

// ---------------------------------------------------------------- geometry --

// One FP32 rotated coordinate, fixed order: fma(m0, x, fma(m1, y, m2*z)).
inline float rot_axis(const float* m, float x, float y, float z) {
  return std::fmaf(m[0], x, std::fmaf(m[1], y, m[2] * z));
}

struct VoxelPos {
  float u[3];  // continuous voxel coordinate; voxel k is centred at u == k
};

// u = side/2 + 0.5 + R.c  (emc_cuda.cu:86-88 before rounding)
inline VoxelPos voxel_pos(const float* m, int side, float x, float y, float z) {
  const float c = (float)side / 2.0f + 0.5f;
  VoxelPos p;
  p.u[0] = c + rot_axis(m + 0, x, y, z);
  p.u[1] = c + rot_axis(m + 3, x, y, z);
  p.u[2] = c + rot_axis(m + 6, x, y, z);
  return p;
}

// Gathers/scatters of one pixel: up to 8 (voxel, weight) pairs.
struct Stencil {
  int n;
  int64_t v[8];
  double w[8];
};

// lower: 1 -> exclusive lower bound (expand, emc_cuda.cu:89-91),
//        0 -> inclusive lower bound (insert, emc_atomic.cu:56-58).
inline void stencil(const VoxelPos& p, int side, int interp, int lower, Stencil* s) {
  s->n = 0;
  if (interp == ORC_NEAREST) {
    int k[3];
    for (int a = 0; a < 3; ++a) {
      k[a] = (int)std::roundf(p.u[a]);
      if (k[a] < lower || k[a] >= side) return;
    }
    s->v[0] = ((int64_t)k[2] * side + k[1]) * side + k[0];
    s->w[0] = 1.0;
    s->n = 1;
    return;
  }
  // trilinear: corners floor(u), floor(u)+1; each corner inside [0, side)
  int k0[3];
  double f[3];
  for (int a = 0; a < 3; ++a) {
    float fl = std::floor(p.u[a]);
    k0[a] = (int)fl;
    f[a] = (double)p.u[a] - (double)fl;
  }
  for (int c = 0; c < 8; ++c) {
    int k[3];
    double w = 1.0;
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      int b = (c >> a) & 1;
      k[a] = k0[a] + b;
      w *= b ? f[a] : 1.0 - f[a];
      if (k[a] < 0 || k[a] >= side) ok = false;
    }
    if (!ok || w == 0.0) continue;
    s->v[s->n] = ((int64_t)k[2] * side + k[1]) * side + k[0];
    s->w[s->n] = w;
    s->n++;
  }
}

std::vector<int64_t> active_pixels(const int32_t* mask, int64_t npix, bool insert_rule) {
  std::vector<int64_t> a;
  for (int64_t i = 0; i < npix; ++i)
    if (insert_rule ? mask[i] == 1 : mask[i] != 0) a.push_back(i);
  return a;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------- rotations --

int64_t orc_n_to_samples(int n) { return 20 * ((int64_t)n + 5 * (int64_t)n * n * n); }

void orc_rotation_matrix_f32(const float* q, float* m) {
  // emc_cuda.cu:65-85 coefficients, each product rounded (no contraction).
  const float q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
  m[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
  m[1] = 2.0f * q1 * q2 - 2.0f * q0 * q3;
  m[2] = 2.0f * q1 * q3 + 2.0f * q0 * q2;
  m[3] = 2.0f * q1 * q2 + 2.0f * q0 * q3;
  m[4] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
  m[5] = 2.0f * q2 * q3 - 2.0f * q0 * q1;
  m[6] = 2.0f * q1 * q3 - 2.0f * q0 * q2;
  m[7] = 2.0f * q2 * q3 + 2.0f * q0 * q1;
  m[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
}

int64_t orc_generate_rotations(int n, int halve, double* q_out, double* w_out) {
  // emc.c:40-41: golden ratio with sqrt(5) written as 2.23606798
  const double tau = (1.0 + 2.23606798) / 2.0;
  const int64_t total = orc_n_to_samples(n);
  if (n < 1) return 0;
  if (!q_out || !w_out) return halve ? total / 2 : total;

  // 120 vertices of the 600-cell (emc.c:52-103)
  double v[120][4];
  std::memset(v, 0, sizeof(v));
  for (int i = 0; i < 16; ++i)
    for (int k = 0; k < 4; ++k) v[i][k] = -0.5 + ((i >> (3 - k)) & 1);
  for (int i = 0; i < 8; ++i) v[16 + i][i / 2] = -1.0 + 2.0 * (i % 2);
  static const int perm[12][4] = {{1, 2, 3, 4}, {1, 4, 2, 3}, {1, 3, 4, 2}, {2, 3, 1, 4},
                                  {2, 4, 3, 1}, {2, 1, 4, 3}, {3, 1, 2, 4}, {3, 4, 1, 2},
                                  {3, 2, 4, 1}, {4, 2, 1, 3}, {4, 3, 2, 1}, {4, 1, 3, 2}};
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 8; ++j) {
      const int j1 = (j >> 2) & 1, j2 = (j >> 1) & 1, j3 = j & 1;
      double* t = v[24 + 8 * i + j];
      t[perm[i][0] - 1] = -0.5 + j1;
      t[perm[i][1] - 1] = tau * (-0.5 + j2);
      t[perm[i][2] - 1] = (1.0 / tau) * (-0.5 + j3);
      t[perm[i][3] - 1] = 0.0;
    }
  auto norm2sum = [&](std::initializer_list<int> ids) {
    double s = 0;
    for (int k = 0; k < 4; ++k) {
      double a = 0;
      for (int id : ids) a += v[id][k];
      s += a * a;
    }
    return s;
  };
  // edges: |vi+vj|^2 > 3 (emc.c:105-129), j < i.  Pairs with vi.vj == 1/2 sit
  // exactly on the cut; the reference's float arithmetic puts all of them at or
  // below 3 (it finds 720 edges), so the FP64 test carries an explicit margin.
  std::vector<std::array<int, 2>> edges;
  for (int i = 0; i < 120; ++i)
    for (int j = 0; j < i; ++j)
      if (norm2sum({i, j}) > 3.0 + 1e-6) edges.push_back({i, j});
  // faces: edge + vertex not yet used as an edge endpoint, > 7.5 (emc.c:131-168)
  std::vector<std::array<int, 3>> faces;
  {
    bool done[120] = {false};
    for (auto& e : edges) {
      done[e[0]] = done[e[1]] = true;
      for (int j = 0; j < 120; ++j) {
        if (done[j]) continue;
        if (norm2sum({j, e[0], e[1]}) > 7.5) faces.push_back({e[0], e[1], j});
      }
    }
  }
  // cells: vertex j (in order) + face with no vertex already used, > 13.5 (emc.c:170-210)
  std::vector<std::array<int, 4>> cells;
  {
    bool done[120] = {false};
    for (int j = 0; j < 120; ++j) {
      done[j] = true;
      for (auto& f : faces) {
        if (done[f[0]] || done[f[1]] || done[f[2]]) continue;
        if (norm2sum({f[0], f[1], f[2], j}) > 13.5) cells.push_back({f[0], f[1], f[2], j});
      }
    }
  }
  if (edges.size() != 720 || faces.size() != 1200 || cells.size() != 600) return -1;

  // weights (emc.c:212-217)
  const double alpha = std::acos(1.0 / 3.0);
  const double f1 = 5.0 * alpha / 2.0 / M_PI;
  const double f0 = 20.0 * (3.0 * alpha - M_PI) / 4.0 / M_PI;
  const double f2 = 1.0, f3 = 1.0;
  std::vector<std::array<double, 4>> q(total);
  std::vector<double> w(total);
  auto put = [&](int64_t idx, const double* p, double f) {
    for (int k = 0; k < 4; ++k) q[idx][k] = p[k];
    const double r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
    w[idx] = f / (double)total / std::pow(r2, 1.5);
  };
  for (int i = 0; i < 120; ++i) put(i, v[i], f0);
  const int ev = n - 1;  // points per edge
  const int64_t edges_base = 120;
  for (int i = 0; i < 720; ++i)
    for (int j = 0; j < ev; ++j) {  // emc.c:247-259
      double p[4];
      for (int k = 0; k < 4; ++k)
        p[k] = (double)(j + 1) / (ev + 1) * v[edges[i][0]][k] +
               (double)(ev - j) / (ev + 1) * v[edges[i][1]][k];
      put(edges_base + (int64_t)ev * i + j, p, f1);
    }
  const int fv = ((n - 1) * (n - 2)) / 2;
  const int64_t faces_base = 120 + 720 * (int64_t)ev;
  if (fv > 0)
    for (int i = 0; i < 1200; ++i) {  // emc.c:267-294
      int count = 0;
      for (int ka = 2; ka < ev + 1; ++ka)
        for (int kb = 2; kb < ev + 1; ++kb) {
          if (ka + kb <= ev + 1) continue;
          const int kc = 2 * (ev + 1) - ka - kb;
          const double den = 3 * (ev + 1) - ka - kb - kc;
          const double a = (ev + 1 - ka) / den, b = (ev + 1 - kb) / den, c = (ev + 1 - kc) / den;
          double p[4];
          for (int k = 0; k < 4; ++k)
            p[k] = a * v[faces[i][0]][k] + b * v[faces[i][1]][k] + c * v[faces[i][2]][k];
          put(faces_base + (int64_t)fv * i + count, p, f2);
          count++;
        }
    }
  const int cv = ((n - 1) * (n - 2) * (n - 3)) / 6;
  const int64_t cell_base = faces_base + 1200 * (int64_t)fv;
  if (cv > 0)
    for (int i = 0; i < 600; ++i) {  // emc.c:303-334
      int count = 0;
      for (int ka = 3; ka < ev + 1; ++ka)
        for (int kb = 3; kb < ev + 1; ++kb)
          for (int kc = 3; kc < ev + 1; ++kc) {
            const int kd = 3 * (ev + 1) - ka - kb - kc;
            if (kd < 3 || kd >= ev + 1) continue;
            const double den = 4 * (ev + 1) - ka - kb - kc - kd;
            const double a = (ev + 1 - ka) / den, b = (ev + 1 - kb) / den;
            const double c = (ev + 1 - kc) / den, d = (ev + 1 - kd) / den;
            double p[4];
            for (int k = 0; k < 4; ++k)
              p[k] = a * v[cells[i][0]][k] + b * v[cells[i][1]][k] + c * v[cells[i][2]][k] +
                     d * v[cells[i][3]][k];
            put(cell_base + (int64_t)cv * i + count, p, f3);
            count++;
          }
    }
  // normalise weights, then quaternions (emc.c:337-359)
  double ws = 0;
  for (double x : w) ws += x;
  for (double& x : w) x /= ws;
  for (auto& p : q) {
    const double r = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
    for (int k = 0; k < 4; ++k) p[k] /= r;
  }
  int64_t out = 0;
  double kept_w = 0;
  for (int64_t i = 0; i < total; ++i) {
    if (halve) {
      // keep the member of the +-q pair whose first non-zero component is positive
      int k = 0;
      while (k < 3 && q[i][k] == 0.0) ++k;
      if (!(q[i][k] > 0.0)) continue;
    }
    for (int k = 0; k < 4; ++k) q_out[4 * out + k] = q[i][k];
    w_out[out] = w[i];
    kept_w += w[i];
    out++;
  }
  for (int64_t i = 0; i < out; ++i) w_out[i] /= kept_w;
  return out;
}

void orc_coordinates(int side, double wavelength, double pixel_size, double detector_distance,
                     double* xo, double* yo, double* zo) {
  // emc.c:365-393, stored at [y*side + x]
  for (int x = 0; x < side; ++x)
    for (int y = 0; y < side; ++y) {
      const double px = (double)(x - side / 2) + 0.5;
      const double py = (double)(y - side / 2) + 0.5;
      const double pr = std::sqrt(px * px + py * py);
      const double ang = std::atan2(pr * pixel_size, detector_distance);
      const double fr = std::sin(ang) / wavelength;
      const double fz = (1.0 - std::cos(ang)) / wavelength;
      const int64_t i = (int64_t)y * side + x;
      xo[i] = px;
      yo[i] = py;
      zo[i] = fz / fr * pr;
    }
}

// ---------------------------------------------------------------- expand --

void orc_expand(const orc_config* c, const double* model, const float* rot, const float* cx,
                const float* cy, const float* cz, double* slices) {
  const int side = c->side;
  const int64_t npix = (int64_t)side * side;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t r = 0; r < c->n_rotations; ++r) {
    float m[9];
    orc_rotation_matrix_f32(rot + 4 * r, m);
    double* s = slices + r * npix;
    for (int64_t i = 0; i < npix; ++i) {
      VoxelPos p = voxel_pos(m, side, cx[i], cy[i], cz[i]);
      Stencil st;
      stencil(p, side, c->interp, c->interp == ORC_NEAREST ? 1 : 0, &st);
      double acc = 0;
      for (int k = 0; k < st.n; ++k) acc += st.w[k] * model[st.v[k]];
      s[i] = acc;
    }
  }
}

// -------------------------------------------------------- log-likelihood --

// One dot product in a fixed order: four partial sums over j = 0, 1, 2, 3
// (mod 4), the tail added to the first, combined as (s0 + s1) + (s2 + s3).
static inline double dot4(const double* a, const double* b, int64_t P) {
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int64_t j = 0;
  for (; j + 4 <= P; j += 4) {
    s0 += a[j] * b[j];
    s1 += a[j + 1] * b[j + 1];
    s2 += a[j + 2] * b[j + 2];
    s3 += a[j + 3] * b[j + 3];
  }
  for (; j < P; ++j) s0 += a[j] * b[j];
  return (s0 + s1) + (s2 + s3);
}

typedef double v4d __attribute__((vector_size(32)));

static inline v4d load4(const double* p) {
  v4d v;
  std::memcpy(&v, p, sizeof(v));
  return v;
}

// C[r][p] = sum_{active j} A[r][j] * B[p][j] in FP64.  Blocks of 16 r x 64 p
// walk j in chunks of 256 (the block's rows of a chunk stay in L1/L2); 2 x 4
// sub-blocks share their loads.  Lane k of each vector accumulator is dot4's
// partial sum k, carried across the chunks in j order, so every element is
// summed exactly as dot4 sums it.
static void cross(int64_t R, int64_t N, int64_t P, const double* A, const double* B, double* C) {
  const int64_t RB = 16, NB = 64, JB = 256;
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int64_t r0 = 0; r0 < R; r0 += RB)
    for (int64_t p0 = 0; p0 < N; p0 += NB) {
      const int64_t r1 = std::min(R, r0 + RB), p1 = std::min(N, p0 + NB);
      const int64_t P4 = P / 4 * 4;
      const int64_t rq = r0 + (r1 - r0) / 2 * 2, pq = p0 + (p1 - p0) / 4 * 4;
      v4d acc[RB][NB];
      for (int64_t r = r0; r < rq; ++r)
        for (int64_t p = p0; p < pq; ++p) acc[r - r0][p - p0] = v4d{0, 0, 0, 0};
      for (int64_t j0 = 0; j0 < P4; j0 += JB) {
        const int64_t j1 = std::min(P4, j0 + JB);
        for (int64_t r = r0; r < rq; r += 2) {
          const double* a0 = A + r * P;
          const double* a1 = a0 + P;
          for (int64_t p = p0; p < pq; p += 4) {
            const double* b0 = B + p * P;
            const double* b1 = b0 + P;
            const double* b2 = b1 + P;
            const double* b3 = b2 + P;
            v4d* s0 = &acc[r - r0][p - p0];
            v4d* s1 = &acc[r + 1 - r0][p - p0];
            v4d t00 = s0[0], t01 = s0[1], t02 = s0[2], t03 = s0[3];
            v4d t10 = s1[0], t11 = s1[1], t12 = s1[2], t13 = s1[3];
            for (int64_t j = j0; j < j1; j += 4) {
              const v4d x0 = load4(a0 + j), x1 = load4(a1 + j);
              const v4d y0 = load4(b0 + j), y1 = load4(b1 + j), y2 = load4(b2 + j),
                        y3 = load4(b3 + j);
              t00 += x0 * y0; t01 += x0 * y1; t02 += x0 * y2; t03 += x0 * y3;
              t10 += x1 * y0; t11 += x1 * y1; t12 += x1 * y2; t13 += x1 * y3;
            }
            s0[0] = t00; s0[1] = t01; s0[2] = t02; s0[3] = t03;
            s1[0] = t10; s1[1] = t11; s1[2] = t12; s1[3] = t13;
          }
        }
      }
      for (int64_t r = r0; r < rq; ++r)
        for (int64_t p = p0; p < pq; ++p) {
          const v4d s = acc[r - r0][p - p0];
          double l0 = s[0];
          for (int64_t j = P4; j < P; ++j) l0 += A[r * P + j] * B[p * P + j];
          C[r * N + p] = (l0 + s[1]) + (s[2] + s[3]);
        }
      // the ragged edges of the block, one element at a time
      for (int64_t r = r0; r < r1; ++r)
        for (int64_t p = (r < rq ? pq : p0); p < p1; ++p)
          C[r * N + p] = dot4(A + r * P, B + p * P, P);
    }
}

void orc_loglik(const orc_config* c, const double* slices, const float* images,
                const int32_t* mask, const double* scaling, double* ll) {
  const int64_t R = c->n_rotations, N = c->n_patterns;
  const int64_t npix = (int64_t)c->side * c->side;
  const std::vector<int64_t> act = active_pixels(mask, npix, false);
  const int64_t P = (int64_t)act.size();
  std::vector<double> A(R * P), B(N * P), rowA(R, 0.0), rowB(N, 0.0);
  const bool gauss = c->likelihood == ORC_LL_GAUSS;
#pragma omp parallel for
  for (int64_t r = 0; r < R; ++r)
    for (int64_t j = 0; j < P; ++j) {
      const double s = slices[r * npix + act[j]];
      // gauss: cross term S.K, rowA = sum S^2;  poisson: K.log W, rowA = sum W
      A[r * P + j] = gauss ? s : std::log(std::max(s, c->poisson_floor));
      rowA[r] += gauss ? s * s : s;
    }
#pragma omp parallel for
  for (int64_t p = 0; p < N; ++p)
    for (int64_t j = 0; j < P; ++j) {
      const double k = images[p * npix + act[j]];
      B[p * P + j] = k;
      rowB[p] += k * k;
    }
  cross(R, N, P, A.data(), B.data(), ll);
  const double inv = 1.0 / (2.0 * (double)P * c->sigma * c->sigma);
#pragma omp parallel for
  for (int64_t r = 0; r < R; ++r)
    for (int64_t p = 0; p < N; ++p) {
      const double x = ll[r * N + p], phi = scaling[p];
      // gauss: -(sum S^2 - 2/phi sum S K + 1/phi^2 sum K^2) / (2 cnt sigma^2)
      ll[r * N + p] = gauss ? -(rowA[r] - 2.0 * x / phi + rowB[p] / (phi * phi)) * inv
                            : x - phi * rowA[r];
    }
}

void orc_loglik_gauss_direct(const orc_config* c, const double* slices, const float* images,
                             const int32_t* mask, const double* scaling, double* ll) {
  // emc.c:668-682 / emc_cuda.cu:114-149 literally, in FP64.
  const int64_t R = c->n_rotations, N = c->n_patterns;
  const int64_t npix = (int64_t)c->side * c->side;
#pragma omp parallel for collapse(2)
  for (int64_t r = 0; r < R; ++r)
    for (int64_t p = 0; p < N; ++p) {
      double sum = 0;
      int64_t cnt = 0;
      for (int64_t i = 0; i < npix; ++i)
        if (mask[i] != 0) {
          const double d = slices[r * npix + i] - images[p * npix + i] / scaling[p];
          sum += d * d;
          cnt++;
        }
      ll[r * N + p] = -sum / 2.0 / (double)cnt / (c->sigma * c->sigma);
    }
}

// --------------------------------------------------------------- softmax --

double orc_softmax(int64_t R, int64_t N, double* resp, double* lse) {
  double plogp = 0;
#pragma omp parallel for reduction(+ : plogp)
  for (int64_t p = 0; p < N; ++p) {
    double mx = -INFINITY;
    for (int64_t r = 0; r < R; ++r) mx = std::max(mx, resp[r * N + p]);
    double s = 0;
    for (int64_t r = 0; r < R; ++r) {
      const double e = std::exp(resp[r * N + p] - mx);
      resp[r * N + p] = e;
      s += e;
    }
    for (int64_t r = 0; r < R; ++r) {
      const double P = resp[r * N + p] / s;
      resp[r * N + p] = P;
      if (P > 0) plogp += P * std::log(P);
    }
    if (lse) lse[p] = mx + std::log(s);
  }
  return plogp;
}

// --------------------------------------------------------------- scaling --

void orc_update_scaling(const orc_config* c, const double* slices, const float* images,
                        const int32_t* mask, const double* resp, double* scaling) {
  const int64_t R = c->n_rotations, N = c->n_patterns;
  const int64_t npix = (int64_t)c->side * c->side;
  const std::vector<int64_t> act = active_pixels(mask, npix, false);
  const int64_t P = (int64_t)act.size();
  const bool gauss = c->likelihood == ORC_LL_GAUSS;
  std::vector<double> num(N, 0.0), den(N, 0.0);
  if (gauss) {
    // emc_cuda.cu:195-228: phi = sum K^2 / sum_r P_rp sum K S_r
    std::vector<double> A(R * P), B(N * P), C(R * N);
#pragma omp parallel for
    for (int64_t r = 0; r < R; ++r)
      for (int64_t j = 0; j < P; ++j) A[r * P + j] = slices[r * npix + act[j]];
#pragma omp parallel for
    for (int64_t p = 0; p < N; ++p)
      for (int64_t j = 0; j < P; ++j) {
        const double k = images[p * npix + act[j]];
        B[p * P + j] = k;
        num[p] += k * k;
      }
    cross(R, N, P, A.data(), B.data(), C.data());
#pragma omp parallel for
    for (int64_t p = 0; p < N; ++p) {
      double d = 0;
      for (int64_t r = 0; r < R; ++r) d += resp[r * N + p] * C[r * N + p];
      den[p] = d;
    }
  } else {
    // poisson MLE: phi = sum K / sum_r P_rp sum W_r
    std::vector<double> sw(R, 0.0);
#pragma omp parallel for
    for (int64_t r = 0; r < R; ++r)
      for (int64_t j = 0; j < P; ++j) sw[r] += slices[r * npix + act[j]];
#pragma omp parallel for
    for (int64_t p = 0; p < N; ++p) {
      double k = 0, d = 0;
      for (int64_t j = 0; j < P; ++j) k += images[p * npix + act[j]];
      for (int64_t r = 0; r < R; ++r) d += resp[r * N + p] * sw[r];
      num[p] = k;
      den[p] = d;
    }
  }
  for (int64_t p = 0; p < N; ++p)
    if (num[p] > 0 && den[p] > 0) scaling[p] = num[p] / den[p];
}

// -------------------------------------------------------------- compress --

void orc_slice_average(const orc_config* c, const double* resp, const float* images,
                       const int32_t* mask, const double* scaling, double* U,
                       double* total_resp) {
  // U[r][i] = sum_p P_rp K_pi / phi_p for mask != 0 (emc_atomic.cu:89-98, emc.c:541-555),
  // T_r = sum_p P_rp; pixels with mask == 0 are left at 0.
  const int64_t R = c->n_rotations, N = c->n_patterns;
  const int64_t npix = (int64_t)c->side * c->side;
  const std::vector<int64_t> act = active_pixels(mask, npix, false);
  const int64_t P = (int64_t)act.size();
  std::vector<double> Kt(P * N), Ua(R * P);
#pragma omp parallel for
  for (int64_t j = 0; j < P; ++j)
    for (int64_t p = 0; p < N; ++p) Kt[j * N + p] = images[p * npix + act[j]] / scaling[p];
  cross(R, P, N, resp, Kt.data(), Ua.data());
#pragma omp parallel for
  for (int64_t r = 0; r < R; ++r) {
    double t = 0;
    for (int64_t p = 0; p < N; ++p) t += resp[r * N + p];
    total_resp[r] = t;
    double* u = U + r * npix;
    for (int64_t i = 0; i < npix; ++i) u[i] = 0.0;
    for (int64_t j = 0; j < P; ++j) u[act[j]] = Ua[r * P + j];
  }
}

void orc_insert(const orc_config* c, const double* U, const double* total_resp,
                const int32_t* mask, const float* rot, const float* rotw, const float* cx,
                const float* cy, const float* cz, double* model_acc, double* weight_acc) {
  orc_insert_shard(c, U, total_resp, total_resp, mask, rot, rotw, cx, cy, cz, model_acc,
                   weight_acc);
}

void orc_insert_shard(const orc_config* c, const double* U, const double* total_resp,
                      const double* all_total_resp, const int32_t* mask, const float* rot,
                      const float* rotw, const float* cx, const float* cy, const float* cz,
                      double* model_acc, double* weight_acc) {
  // emc_atomic.cu:115-133 + :17-73: rotations with T_r <= 1e-10 are skipped;
  // model += w * U/T, weight += w with w = rotw_r * T_r, for mask == 1 pixels.
  // For a shard of the patterns the skip test reads the total over all
  // shards (all_total_resp), so the shards' sums add up to the unsharded one.
  // The rotations are split into a number of contiguous chunks fixed by the
  // shape alone (not by the thread count); each chunk is accumulated serially
  // into its own grids and the chunks are added in order, so the result is
  // the same on every machine.
  const int side = c->side;
  const int64_t npix = (int64_t)side * side;
  const int64_t M = npix * side, R = c->n_rotations;
  const std::vector<int64_t> ins = active_pixels(mask, npix, true);
  const int64_t budget = (int64_t)1 << 29;  // bytes of per-chunk grids
  int64_t nch = std::min<int64_t>(32, std::max<int64_t>(1, budget / (16 * M)));
  nch = std::max<int64_t>(1, std::min<int64_t>(nch, R));
  std::vector<double> part(nch > 1 ? (size_t)(2 * M * nch) : 0, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t ch = 0; ch < nch; ++ch) {
    double* ma = nch > 1 ? part.data() + 2 * M * ch : model_acc;
    double* wa = nch > 1 ? ma + M : weight_acc;
    for (int64_t r = R * ch / nch; r < R * (ch + 1) / nch; ++r) {
      const double T = total_resp[r];
      if (!(all_total_resp[r] > 1e-10) || !(T > 0.0)) continue;
      const double w = (double)rotw[r] * T;
      float m[9];
      orc_rotation_matrix_f32(rot + 4 * r, m);
      for (int64_t i : ins) {
        VoxelPos pos = voxel_pos(m, side, cx[i], cy[i], cz[i]);
        Stencil st;
        stencil(pos, side, c->interp, 0, &st);
        const double s = U[r * npix + i] / T;
        for (int k = 0; k < st.n; ++k) {
          ma[st.v[k]] += st.w[k] * w * s;
          wa[st.v[k]] += st.w[k] * w;
        }
      }
    }
  }
  if (nch > 1) {
#pragma omp parallel for
    for (int64_t v = 0; v < M; ++v)
      for (int64_t ch = 0; ch < nch; ++ch) {
        model_acc[v] += part[2 * M * ch + v];
        weight_acc[v] += part[2 * M * ch + M + v];
      }
  }
}

void orc_compress(const orc_config* c, const double* resp, const float* images,
                  const int32_t* mask, const double* scaling, const float* rot,
                  const float* rotw, const float* cx, const float* cy, const float* cz,
                  double* model_acc, double* weight_acc, double* total_resp) {
  const int64_t npix = (int64_t)c->side * c->side;
  std::vector<double> U(c->n_rotations * npix);
  orc_slice_average(c, resp, images, mask, scaling, U.data(), total_resp);
  orc_insert(c, U.data(), total_resp, mask, rot, rotw, cx, cy, cz, model_acc, weight_acc);
}

void orc_normalize_model(int64_t M, double* model, const double* weight) {
  double sum = 0;
  for (int64_t i = 0; i < M; ++i) {
    model[i] = weight[i] > 0.0 ? model[i] / weight[i] : 0.0;
    sum += model[i];
  }
  const double mean = sum / (double)M;
  if (mean != 0.0)
    for (int64_t i = 0; i < M; ++i) model[i] /= mean;
}

// ------------------------------------------------- synthetic inputs --
// The seeded synthetic datasets of the benchmark configurations, restated
// here so that a CPU-only run (the timed CPU baseline) needs nothing but this
// library.  Same counter-based streams, Poisson sampler and FP32 trilinear
// weights as the engine's host generator, so both produce identical data.

namespace {

inline uint64_t syn_mix(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Draw i of stream (seed, a, b) is a pure function of (seed, a, b, i).
struct SynStream {
  uint64_t key, ctr = 0;
  SynStream(uint64_t seed, uint64_t a, uint64_t b) : key(syn_mix(syn_mix(seed ^ syn_mix(a)) + b)) {}
  double uniform() { return (double)(syn_mix(key + syn_mix(ctr++)) >> 11) * 0x1.0p-53; }
  double normal() {  // Box-Muller, first output
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
  }
  // Inversion for means below 12, else Hormann's PTRS transformed rejection.
  double poisson(double lam) {
    if (!(lam > 0)) return 0.0;
    if (lam < 12.0) {
      double p = std::exp(-lam), s = p, u = uniform();
      int k = 0;
      while (u > s && k < 1000) {
        ++k;
        p *= lam / k;
        s += p;
      }
      return k;
    }
    const double slam = std::sqrt(lam), loglam = std::log(lam);
    const double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4), vr = 0.9277 - 3.6224 / (b - 2.0);
    for (;;) {
      const double U = uniform() - 0.5, V = uniform();
      const double us = 0.5 - std::fabs(U);
      const double k = std::floor((2.0 * a / us + b) * U + lam + 0.43);
      if (us >= 0.07 && V <= vr) return k;
      if (k < 0 || (us < 0.013 && V > us)) continue;
      if (std::log(V) + std::log(invalpha) - std::log(a / (us * us) + b) <=
          -lam + k * loglam - std::lgamma(k + 1.0))
        return k;
    }
  }
};

// Trilinear sample of the model at continuous voxel position u: FP32 corner
// weights (x, y, z factors multiplied in that order), corners in bit order,
// zero-weight and out-of-grid corners skipped, FP64 sum.
double syn_trilinear(const float* model, int side, const float* u) {
  const float fx = std::floor(u[0]), fy = std::floor(u[1]), fz = std::floor(u[2]);
  const float ax = u[0] - fx, ay = u[1] - fy, az = u[2] - fz;
  double acc = 0;
  for (int c = 0; c < 8; ++c) {
    const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
    const int kx = (int)fx + bx, ky = (int)fy + by, kz = (int)fz + bz;
    if (kx < 0 || kx >= side || ky < 0 || ky >= side || kz < 0 || kz >= side) continue;
    const float w = (bx ? ax : 1.0f - ax) * (by ? ay : 1.0f - ay) * (bz ? az : 1.0f - az);
    if (w == 0.0f) continue;
    acc += (double)w * model[((int64_t)kz * side + ky) * side + kx];
  }
  return acc;
}

}  // namespace

void orc_random_model(int side, uint64_t seed, float* model) {
  const int64_t M = (int64_t)side * side * side;
#pragma omp parallel for
  for (int64_t i = 0; i < M; ++i) {
    SynStream s(seed, 0x6d6f64656cull, (uint64_t)i);
    model[i] = (float)s.uniform();
  }
}

int orc_synthesize(int side, int n_scatterers, double object_radius, int64_t n_patterns,
                   double mean_photons, double scale_sigma, double beamstop_radius,
                   uint64_t seed, int64_t first_pattern, const float* x, const float* y,
                   const float* z, float* true_model, float* counts, int32_t* mask) {
  if (side < 2 || n_patterns < 1 || n_scatterers < 1 || first_pattern < 0 || !x || !y || !z ||
      !counts || !mask)
    return 1;
  const int64_t npix = (int64_t)side * side, M = npix * side;
  // unit point scatterers uniform in a sphere of radius object_radius * side
  std::vector<std::array<double, 3>> pos(n_scatterers);
  {
    SynStream s(seed, 0x73636174ull, 0);
    const double rad = object_radius * side;
    for (auto& p : pos) {
      double a, b, c;
      do {
        a = 2 * s.uniform() - 1;
        b = 2 * s.uniform() - 1;
        c = 2 * s.uniform() - 1;
      } while (a * a + b * b + c * c > 1.0);
      p = {a * rad, b * rad, c * rad};
    }
  }
  // |F|^2 at every voxel centre (voxel k at pixel-unit position k - side/2 - 0.5)
  std::vector<float> model(M);
#pragma omp parallel for
  for (int64_t v = 0; v < M; ++v) {
    const int kx = (int)(v % side), ky = (int)((v / side) % side), kz = (int)(v / npix);
    const double qx = kx - side / 2.0 - 0.5, qy = ky - side / 2.0 - 0.5, qz = kz - side / 2.0 - 0.5;
    double re = 0, im = 0;
    for (const auto& p : pos) {
      const double ph = 2.0 * M_PI * (qx * p[0] + qy * p[1] + qz * p[2]) / side;
      re += std::cos(ph);
      im += std::sin(ph);
    }
    model[v] = (float)(re * re + im * im);
  }
  if (true_model) std::memcpy(true_model, model.data(), sizeof(float) * M);
  int64_t active = 0;  // beamstop: pixel centres within the radius are masked
  for (int iy = 0; iy < side; ++iy)
    for (int ix = 0; ix < side; ++ix) {
      const double dx = ix - side / 2.0 + 0.5, dy = iy - side / 2.0 + 0.5;
      const int on = std::sqrt(dx * dx + dy * dy) > beamstop_radius ? 1 : 0;
      mask[(int64_t)iy * side + ix] = on;
      active += on;
    }
  if (active == 0) return 1;
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t p = 0; p < n_patterns; ++p) {
    const uint64_t gp = (uint64_t)(p + first_pattern);
    SynStream s(seed, 0x70617474ull, gp);
    // uniform random rotation (Shoemake), lognormal scale of mean 1
    const double u1 = s.uniform(), u2 = s.uniform(), u3 = s.uniform();
    const float q[4] = {(float)(std::sqrt(1 - u1) * std::sin(2 * M_PI * u2)),
                        (float)(std::sqrt(1 - u1) * std::cos(2 * M_PI * u2)),
                        (float)(std::sqrt(u1) * std::sin(2 * M_PI * u3)),
                        (float)(std::sqrt(u1) * std::cos(2 * M_PI * u3))};
    const double scale = std::exp(scale_sigma * s.normal() - 0.5 * scale_sigma * scale_sigma);
    float m[9];
    orc_rotation_matrix_f32(q, m);
    std::vector<double> sl(npix);
    double tot = 0;
    for (int64_t i = 0; i < npix; ++i) {
      const VoxelPos vp = voxel_pos(m, side, x[i], y[i], z[i]);
      sl[i] = syn_trilinear(model.data(), side, vp.u);
      if (mask[i]) tot += sl[i];
    }
    const double f = tot > 0 ? mean_photons * scale / tot : 0.0;
    SynStream d(seed, 0x636f756eull, gp);
    float* out = counts + p * npix;
    for (int64_t i = 0; i < npix; ++i) out[i] = (float)d.poisson(sl[i] * f);
  }
  return 0;
}

void orc_iterate(const orc_config* c, const float* images, const int32_t* mask, const float* rot,
                 const float* rotw, const float* cx, const float* cy, const float* cz,
                 double* model, double* scaling, double* resp_out, orc_stats* stats) {
  orc_iterate_restricted(c, images, mask, rot, rotw, cx, cy, cz, nullptr, model, scaling,
                         resp_out, stats);
}

void orc_iterate_restricted(const orc_config* c, const float* images, const int32_t* mask,
                            const float* rot, const float* rotw, const float* cx, const float* cy,
                            const float* cz, const uint8_t* allowed, double* model,
                            double* scaling, double* resp_out, orc_stats* stats) {
  const int64_t R = c->n_rotations, N = c->n_patterns;
  const int64_t npix = (int64_t)c->side * c->side;
  const int64_t M = npix * c->side;
  std::vector<double> S(R * npix), P(R * N), lse(N), T(R);
  orc_expand(c, model, rot, cx, cy, cz, S.data());
  orc_loglik(c, S.data(), images, mask, scaling, P.data());
  if (allowed)  // rotations outside a pattern's candidate set get no responsibility
    for (int64_t i = 0; i < R * N; ++i)
      if (!allowed[i]) P[i] = -INFINITY;
  const double plogp = orc_softmax(R, N, P.data(), lse.data());
  orc_update_scaling(c, S.data(), images, mask, P.data(), scaling);
  std::vector<double> wacc(M, 0.0);
  std::fill(model, model + M, 0.0);
  orc_compress(c, P.data(), images, mask, scaling, rot, rotw, cx, cy, cz, model, wacc.data(),
               T.data());
  orc_normalize_model(M, model, wacc.data());
  if (resp_out) std::memcpy(resp_out, P.data(), sizeof(double) * R * N);
  if (stats) {
    stats->sum_plogp = plogp;
    double tl = 0;
    for (int64_t p = 0; p < N; ++p) tl += lse[p];
    stats->total_loglik = tl;
    double mx = 0;
    for (int64_t i = 0; i < M; ++i) mx = std::max(mx, model[i]);
    stats->model_max = mx;
    double tr = 0;
    for (int64_t r = 0; r < R; ++r) tr += T[r];
    stats->total_resp = tr;
  }
}

}  // extern "C"
