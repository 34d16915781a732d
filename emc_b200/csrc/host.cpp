// Host-side input generators of the engine: rotation sampling, detector
// coordinates, seeded synthetic datasets, and the reference's CPU
// insert_slice.  Plain C++17 + OpenMP.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/emc.h"
#include "../../include/emc_b200.h"
#include "voxel.h"

namespace {

// ------------------------------------------------------ counter-based RNG --
// splitmix64 finaliser over (seed, stream, counter): every draw is a pure
// function of its indices, so OpenMP loops generate identical data for any
// thread count.
inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Stream {
  uint64_t key;
  uint64_t ctr = 0;
  Stream(uint64_t seed, uint64_t a, uint64_t b) : key(mix64(mix64(seed ^ mix64(a)) + b)) {}
  double uniform() { return (double)(mix64(key + mix64(ctr++)) >> 11) * 0x1.0p-53; }
  double normal() {  // Box-Muller
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
  }
  // Poisson: inversion by sequential search for small means, PTRS transformed
  // rejection (Hormann 1993, "The transformed rejection method for generating
  // Poisson random variables") otherwise.
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

}  // namespace

extern "C" {

// ---------------------------------------------------------------- rotations --

int64_t emc_n_to_samples(int n) { return 20 * ((int64_t)n + 5 * (int64_t)n * n * n); }

int64_t emc_generate_rotations(int n, int halve, float* quat, float* weights) {
  // 600-cell sampling of emc.c:49-363: 120 vertices; edges, faces and cells
  // found by thresholds on |sum of member vertices|^2; n-1 points per edge,
  // (n-1)(n-2)/2 per face, (n-1)(n-2)(n-3)/6 per cell placed barycentrically;
  // weight f_k / (count * |q|^3), normalised; quaternions normalised.
  if (n < 1) return -1;
  const int64_t total = emc_n_to_samples(n);
  if (!quat || !weights) return halve ? total / 2 : total;
  const double tau = (1.0 + 2.23606798) / 2.0;  // emc.c:41
  std::vector<std::array<double, 4>> v(120, {0, 0, 0, 0});
  for (int i = 0; i < 16; ++i)
    for (int k = 0; k < 4; ++k) v[i][k] = ((i >> (3 - k)) & 1) ? 0.5 : -0.5;
  for (int i = 0; i < 8; ++i) v[16 + i][i / 2] = (i % 2) ? 1.0 : -1.0;
  static const int order[12][4] = {{0, 1, 2, 3}, {0, 3, 1, 2}, {0, 2, 3, 1}, {1, 2, 0, 3},
                                   {1, 3, 2, 0}, {1, 0, 3, 2}, {2, 0, 1, 3}, {2, 3, 0, 1},
                                   {2, 1, 3, 0}, {3, 1, 0, 2}, {3, 2, 1, 0}, {3, 0, 2, 1}};
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 8; ++j) {
      auto& t = v[24 + 8 * i + j];
      t[order[i][0]] = ((j >> 2) & 1) ? 0.5 : -0.5;
      t[order[i][1]] = tau * (((j >> 1) & 1) ? 0.5 : -0.5);
      t[order[i][2]] = (1.0 / tau) * ((j & 1) ? 0.5 : -0.5);
      t[order[i][3]] = 0.0;
    }
  auto sumsq = [&](const int* ids, int m) {
    double s = 0;
    for (int k = 0; k < 4; ++k) {
      double a = 0;
      for (int t = 0; t < m; ++t) a += v[ids[t]][k];
      s += a * a;
    }
    return s;
  };
  std::vector<std::array<int, 2>> edges;
  for (int i = 0; i < 120; ++i)
    for (int j = 0; j < i; ++j) {
      const int ids[2] = {i, j};
      // nearest neighbours give 2+tau = 3.618; the next shell gives exactly 3
      if (sumsq(ids, 2) > 3.0 + 1e-6) edges.push_back({i, j});
    }
  std::vector<std::array<int, 3>> faces;
  {
    std::vector<char> used(120, 0);
    for (const auto& e : edges) {
      used[e[0]] = used[e[1]] = 1;
      for (int j = 0; j < 120; ++j) {
        if (used[j]) continue;
        const int ids[3] = {j, e[0], e[1]};
        if (sumsq(ids, 3) > 7.5) faces.push_back({e[0], e[1], j});
      }
    }
  }
  std::vector<std::array<int, 4>> cells;
  {
    std::vector<char> used(120, 0);
    for (int j = 0; j < 120; ++j) {
      used[j] = 1;
      for (const auto& f : faces) {
        if (used[f[0]] || used[f[1]] || used[f[2]]) continue;
        const int ids[4] = {f[0], f[1], f[2], j};
        if (sumsq(ids, 4) > 13.5) cells.push_back({f[0], f[1], f[2], j});
      }
    }
  }
  if (edges.size() != 720 || faces.size() != 1200 || cells.size() != 600) return -1;

  const double alpha = std::acos(1.0 / 3.0);
  const double fw[4] = {20.0 * (3.0 * alpha - M_PI) / 4.0 / M_PI, 5.0 * alpha / 2.0 / M_PI, 1.0,
                        1.0};
  std::vector<std::array<double, 4>> q(total);
  std::vector<double> w(total);
  int64_t idx = 0;
  auto emit = [&](const double* p, int kind) {
    double r2 = 0;
    for (int k = 0; k < 4; ++k) {
      q[idx][k] = p[k];
      r2 += p[k] * p[k];
    }
    w[idx] = fw[kind] / (double)total / (r2 * std::sqrt(r2));
    ++idx;
  };
  for (int i = 0; i < 120; ++i) emit(v[i].data(), 0);
  const int e1 = n;  // edge_verts + 1
  for (const auto& e : edges)
    for (int j = 0; j < n - 1; ++j) {
      double p[4];
      for (int k = 0; k < 4; ++k)
        p[k] = (double)(j + 1) / e1 * v[e[0]][k] + (double)(n - 1 - j) / e1 * v[e[1]][k];
      emit(p, 1);
    }
  if (n >= 3)
    for (const auto& f : faces)
      for (int ka = 2; ka < e1; ++ka)
        for (int kb = 2; kb < e1; ++kb) {
          if (ka + kb <= e1) continue;
          const int kc = 2 * e1 - ka - kb;
          const double den = 3.0 * e1 - ka - kb - kc;
          double p[4];
          for (int k = 0; k < 4; ++k)
            p[k] = (e1 - ka) / den * v[f[0]][k] + (e1 - kb) / den * v[f[1]][k] +
                   (e1 - kc) / den * v[f[2]][k];
          emit(p, 2);
        }
  if (n >= 4)
    for (const auto& c : cells)
      for (int ka = 3; ka < e1; ++ka)
        for (int kb = 3; kb < e1; ++kb)
          for (int kc = 3; kc < e1; ++kc) {
            const int kd = 3 * e1 - ka - kb - kc;
            if (kd < 3 || kd >= e1) continue;
            const double den = 4.0 * e1 - ka - kb - kc - kd;
            double p[4];
            for (int k = 0; k < 4; ++k)
              p[k] = (e1 - ka) / den * v[c[0]][k] + (e1 - kb) / den * v[c[1]][k] +
                     (e1 - kc) / den * v[c[2]][k] + (e1 - kd) / den * v[c[3]][k];
            emit(p, 3);
          }
  if (idx != total) return -1;
  double wsum = 0;
  for (double x : w) wsum += x;
  int64_t out = 0;
  double kept = 0;
  std::vector<double> wk;
  wk.reserve(halve ? total / 2 : total);
  for (int64_t i = 0; i < total; ++i) {
    const double r = std::sqrt(q[i][0] * q[i][0] + q[i][1] * q[i][1] + q[i][2] * q[i][2] +
                               q[i][3] * q[i][3]);
    double u[4];
    for (int k = 0; k < 4; ++k) u[k] = q[i][k] / r;
    if (halve) {  // q and -q slice identically: keep the one whose first non-zero entry is > 0
      int k = 0;
      while (k < 3 && u[k] == 0.0) ++k;
      if (!(u[k] > 0.0)) continue;
    }
    for (int k = 0; k < 4; ++k) quat[4 * out + k] = (float)u[k];
    wk.push_back(w[i] / wsum);
    kept += w[i] / wsum;
    ++out;
  }
  for (int64_t i = 0; i < out; ++i) weights[i] = (float)(wk[i] / kept);
  return out;
}

void emc_detector_coordinates(int side, double wavelength, double pixel_size,
                              double detector_distance, float* x, float* y, float* z) {
  // emc.c:365-393: in-plane pixel position, z from the Ewald-sphere angle.
  for (int iy = 0; iy < side; ++iy)
    for (int ix = 0; ix < side; ++ix) {
      const double px = (double)(ix - side / 2) + 0.5;
      const double py = (double)(iy - side / 2) + 0.5;
      const double pr = std::sqrt(px * px + py * py);
      const double ang = std::atan2(pr * pixel_size, detector_distance);
      const double qr = std::sin(ang) / wavelength;
      const double qz = (1.0 - std::cos(ang)) / wavelength;
      const int64_t i = (int64_t)iy * side + ix;
      x[i] = (float)px;
      y[i] = (float)py;
      z[i] = (float)(qz / qr * pr);
    }
}

void emc_random_model(int side, uint64_t seed, float* model) {
  const int64_t M = (int64_t)side * side * side;
#pragma omp parallel for
  for (int64_t i = 0; i < M; ++i) {
    Stream s(seed, 0x6d6f64656cull, (uint64_t)i);
    model[i] = (float)s.uniform();
  }
}

emc_status emc_synthesize(const emc_synth_config* sc, const float* x, const float* y,
                          const float* z, float* true_model, float* counts, int32_t* mask,
                          float* true_rot, float* true_scale) {
  if (!sc || !x || !y || !z || !counts || !mask || sc->side < 2 || sc->n_patterns < 1 ||
      sc->n_scatterers < 1 || sc->first_pattern < 0)
    return EMC_ERR_ARG;
  const int side = sc->side;
  const int64_t npix = (int64_t)side * side, M = npix * side, N = sc->n_patterns;
  // point scatterers uniform in a sphere of radius object_radius * side
  std::vector<std::array<double, 3>> pos(sc->n_scatterers);
  {
    Stream s(sc->seed, 0x73636174ull, 0);
    const double rad = sc->object_radius * side;
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
  // |F|^2 at every voxel centre; voxel k is centred at pixel-unit position k - side/2 - 0.5
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
  // beamstop mask (pixel-centre distance <= radius -> 0)
  int64_t active = 0;
  for (int iy = 0; iy < side; ++iy)
    for (int ix = 0; ix < side; ++ix) {
      const double dx = ix - side / 2.0 + 0.5, dy = iy - side / 2.0 + 0.5;
      const int on = std::sqrt(dx * dx + dy * dy) > sc->beamstop_radius ? 1 : 0;
      mask[(int64_t)iy * side + ix] = on;
      active += on;
    }
  if (active == 0) return EMC_ERR_ARG;
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t p = 0; p < N; ++p) {
    const uint64_t gp = (uint64_t)(p + sc->first_pattern);  // index in the whole dataset
    Stream s(sc->seed, 0x70617474ull, gp);
    // uniform random rotation (Shoemake's subgroup algorithm)
    const double u1 = s.uniform(), u2 = s.uniform(), u3 = s.uniform();
    float q[4] = {(float)(std::sqrt(1 - u1) * std::sin(2 * M_PI * u2)),
                  (float)(std::sqrt(1 - u1) * std::cos(2 * M_PI * u2)),
                  (float)(std::sqrt(u1) * std::sin(2 * M_PI * u3)),
                  (float)(std::sqrt(u1) * std::cos(2 * M_PI * u3))};
    const double scale = std::exp(sc->scale_sigma * s.normal() - 0.5 * sc->scale_sigma * sc->scale_sigma);
    float m[9];
    emc_voxel::rotation_matrix(q, m);
    std::vector<double> sl(npix);
    double tot = 0;
    for (int64_t i = 0; i < npix; ++i) {
      float u[3];
      emc_voxel::position(m, side, x[i], y[i], z[i], u);
      double acc = 0;
      int64_t vv[8];
      float ww[8];
      const int nc = emc_voxel::trilinear(u, side, vv, ww);
      for (int c = 0; c < nc; ++c) acc += (double)ww[c] * model[vv[c]];
      sl[i] = acc;
      if (mask[i]) tot += acc;
    }
    const double f = tot > 0 ? sc->mean_photons * scale / tot : 0.0;
    Stream d(sc->seed, 0x636f756eull, gp);
    float* out = counts + p * npix;
    for (int64_t i = 0; i < npix; ++i) out[i] = (float)d.poisson(sl[i] * f);
    if (true_rot)
      for (int k = 0; k < 4; ++k) true_rot[4 * p + k] = q[k];
    if (true_scale) true_scale[p] = (float)scale;
  }
  return EMC_OK;
}

// ------------------------------------------------ model initialisation ---

emc_status emc_model_random_orientations(int side, int64_t n_images, const float* images,
                                         const int32_t* mask, const float* x, const float* y,
                                         const float* z, uint64_t seed, float* model,
                                         float* quat_out) {
  // emc.c:896-914 (model_input == 1): every image inserted with weight 1 at a
  // uniformly random rotation (Shoemake's subgroup algorithm, as
  // quaternion_random emc.c:27-38), nearest voxel with the insertion bound,
  // mask == 1 pixels; then model = sum / weight, 0 where no weight.
  if (side < 2 || n_images < 0 || (n_images && !images) || !mask || !x || !y || !z || !model)
    return EMC_ERR_ARG;
  const int64_t npix = (int64_t)side * side, M = npix * side;
  std::vector<double> acc(M, 0.0), wt(M, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t p = 0; p < n_images; ++p) {
    Stream s(seed, 0x726f7469ull, (uint64_t)p);
    const double u1 = s.uniform(), u2 = s.uniform(), u3 = s.uniform();
    float q[4] = {(float)(std::sqrt(1 - u1) * std::sin(2 * M_PI * u2)),
                  (float)(std::sqrt(1 - u1) * std::cos(2 * M_PI * u2)),
                  (float)(std::sqrt(u1) * std::sin(2 * M_PI * u3)),
                  (float)(std::sqrt(u1) * std::cos(2 * M_PI * u3))};
    if (quat_out)
      for (int k = 0; k < 4; ++k) quat_out[4 * p + k] = q[k];
    float m[9];
    emc_voxel::rotation_matrix(q, m);
    const float* img = images + p * npix;
    for (int64_t i = 0; i < npix; ++i) {
      if (mask[i] != 1) continue;
      float u[3];
      emc_voxel::position(m, side, x[i], y[i], z[i], u);
      int64_t v;
      if (!emc_voxel::nearest(u, side, 0, &v)) continue;
#pragma omp atomic
      acc[v] += (double)img[i];
#pragma omp atomic
      wt[v] += 1.0;
    }
  }
  for (int64_t v = 0; v < M; ++v) model[v] = wt[v] > 0.0 ? (float)(acc[v] / wt[v]) : 0.0f;
  return EMC_OK;
}

emc_status emc_model_load(const char* path, int side, float* model) {
  // emc.c:915-925 (model_input == 2) reads |value| of a side^3 image; here the
  // file is raw little-endian float32 in [z][y][x] order.
  if (!path || side < 2 || !model) return EMC_ERR_ARG;
  const int64_t M = (int64_t)side * side * side;
  FILE* f = std::fopen(path, "rb");
  if (!f) return EMC_ERR_ARG;
  std::fseek(f, 0, SEEK_END);
  const long bytes = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (bytes != (long)(M * 4)) {
    std::fclose(f);
    return EMC_ERR_RANGE;
  }
  const size_t got = std::fread(model, 4, (size_t)M, f);
  std::fclose(f);
  if (got != (size_t)M) return EMC_ERR_ARG;
  for (int64_t i = 0; i < M; ++i) model[i] = std::fabs(model[i]);
  return EMC_OK;
}

emc_status emc_model_save(const char* path, int side, const float* model) {
  if (!path || side < 2 || !model) return EMC_ERR_ARG;
  const int64_t M = (int64_t)side * side * side;
  FILE* f = std::fopen(path, "wb");
  if (!f) return EMC_ERR_ARG;
  const size_t put = std::fwrite(model, 4, (size_t)M, f);
  const int rc = std::fclose(f);
  return (put == (size_t)M && rc == 0) ? EMC_OK : EMC_ERR_ARG;
}

// ------------------------------------------------- reference CPU routine ---

void insert_slice(sp_3matrix* model, sp_3matrix* weight, sp_matrix* slice, sp_imatrix* mask,
                  real w, Quaternion* rot, sp_matrix* xc, sp_matrix* yc, sp_matrix* zc) {
  // emc.c:491-539: nearest voxel, inclusive lower bound, mask == 1 only.
  const int side = (int)model->x;
  const int64_t npix = (int64_t)slice->rows * slice->cols;
  float m[9];
  emc_voxel::rotation_matrix(rot->q, m);
  for (int64_t i = 0; i < npix; ++i) {
    if (mask->data[i] != 1) continue;
    float u[3];
    emc_voxel::position(m, side, xc->data[i], yc->data[i], zc->data[i], u);
    int64_t v;
    if (!emc_voxel::nearest(u, side, 0, &v)) continue;
    model->data[v] += w * slice->data[i];
    weight->data[v] += w;
  }
}

}  // extern "C"
