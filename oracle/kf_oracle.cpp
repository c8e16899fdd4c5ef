/*
 * kf_oracle.cpp — FP64 CPU oracle (test infrastructure; see kf_oracle.h).
 *
 * A scalar FP64 restatement of the reference's KinectFusion compute path, one function
 * per shader / host routine, each citing the reference file:line it follows.  OpenMP
 * parallelises over image rows and volume columns; every reduction is summed per row
 * and then over rows in row order, so results do not depend on the thread count.
 *
 * Deliberate differences from the reference's FP32 arithmetic:
 *   - everything is FP64, including poses (the reference keeps glm float mat4);
 *   - the integrate z-march and the raycast march evaluate positions directly
 *     (base + k*step) instead of by repeated float addition (integrate.cs:62,
 *     raycast.cs:185) — identical in exact arithmetic;
 *   - the ICP normal equations are solved by a symmetric Jacobi eigen pseudo-inverse,
 *     which is what Eigen::JacobiSVD::solve computes for a symmetric matrix
 *     (gFusion.cpp:696-697); the SDF step uses an unpivoted LDL^T (gFusion.cpp:902).
 */
#include "kf_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#define KF_MC_TABLE_QUAL static const
#include "../oglfusionkinectv2_b200/csrc/generated/kf_mc_tables.inc"

namespace {

constexpr double kShortToF = (double)0.00003051944088f; /* raycast.cs:81 etc. */

/* ---------------- small matrix helpers (column-major 4x4, glm layout) ---------------- */
inline double& M(double* m, int col, int row) { return m[col * 4 + row]; }
inline double Mc(const double* m, int col, int row) { return m[col * 4 + row]; }

void mat4_mul(const double* a, const double* b, double* out) {
  double r[16];
  for (int c = 0; c < 4; ++c)
    for (int rr = 0; rr < 4; ++rr) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += Mc(a, k, rr) * Mc(b, c, k);
      r[c * 4 + rr] = s;
    }
  std::memcpy(out, r, sizeof(r));
}

/* General 4x4 inverse (glm::inverse semantics) by cofactors. */
void mat4_inverse(const double* m, double* out) {
  double inv[16];
  inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] +
           m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] -
           m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] +
           m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] -
            m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] -
           m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] +
           m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] -
           m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] +
            m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] +
           m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] -
           m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] +
            m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] -
            m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] -
           m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] +
           m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] -
            m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] +
            m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
  double id = 1.0 / det;
  for (int i = 0; i < 16; ++i) out[i] = inv[i] * id;
}

/* y = M * (x, w) for the first three rows. */
inline void xform(const double* m, const double* x, double w, double* y) {
  for (int r = 0; r < 3; ++r)
    y[r] = Mc(m, 0, r) * x[0] + Mc(m, 1, r) * x[1] + Mc(m, 2, r) * x[2] + Mc(m, 3, r) * w;
}

/* getCameraMatrix / getInverseCameraMatrix (gFusion.h:451-470) for k = (fx,fy,cx,cy). */
void camera_matrix(double fx, double fy, double cx, double cy, double* K) {
  std::memset(K, 0, 16 * sizeof(double));
  M(K, 0, 0) = fx; M(K, 2, 0) = cx;
  M(K, 1, 1) = fy; M(K, 2, 1) = cy;
  M(K, 2, 2) = 1; M(K, 3, 3) = 1;
}

/* ---------------- IEEE half from double, round to nearest even ---------------------- */
uint16_t half_from_double(double v) {
  uint16_t sign = std::signbit(v) ? 0x8000 : 0;
  double a = std::fabs(v);
  if (std::isnan(v)) return 0x7e00;
  if (a >= 65520.0) return sign | 0x7c00;
  if (a == 0.0) return sign;
  int e2;
  std::frexp(a, &e2);   /* a = m * 2^e2, m in [0.5,1) */
  int e = e2 - 1;       /* a in [2^e, 2^(e+1)) */
  if (e < -14) {        /* subnormal: units of 2^-24 */
    double q = std::nearbyint(std::ldexp(a, 24));
    return sign | (uint16_t)q; /* q == 1024 becomes the smallest normal */
  }
  double q = std::nearbyint(std::ldexp(a, 10 - e)); /* in [1024, 2048] */
  if (q >= 2048.0) { q = 1024.0; ++e; }
  if (e + 15 >= 31) return sign | 0x7c00;
  return sign | (uint16_t)(((e + 15) << 10) | ((int)q - 1024));
}

double half_to_double(uint16_t h) {
  int s = h >> 15, e = (h >> 10) & 31, m = h & 1023;
  double v;
  if (e == 0) v = std::ldexp((double)m, -24);
  else if (e == 31) v = m ? NAN : INFINITY;
  else v = std::ldexp((double)(m + 1024), e - 25);
  return s ? -v : v;
}

/* ---------------- volume with the CUDA path's byte layout ----------------------------
 * Two planes: all TSDF values (x fastest), then all weights.  F32F32: float + float;
 * F16U16: IEEE half + uint16; RG16I: int16 (F*32766, integrate.cs:48) + int16. */
struct Volume {
  int storage = KF_STORAGE_F32F32;
  int nx = 0, ny = 0, nz = 0;
  std::vector<uint8_t> buf;

  size_t count() const { return (size_t)nx * ny * nz; }
  size_t value_bytes() const { return storage == KF_STORAGE_F32F32 ? 4 : 2; }
  size_t bytes() const { return count() * value_bytes() * 2; }
  void alloc(int s, int x, int y, int z) {
    storage = s; nx = x; ny = y; nz = z;
    buf.assign(bytes(), 0u);
  }
  void zero() { std::fill(buf.begin(), buf.end(), 0u); }
  size_t idx(int x, int y, int z) const { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); }
  const uint8_t* fplane() const { return buf.data(); }
  const uint8_t* wplane() const { return buf.data() + count() * value_bytes(); }
  uint8_t* fplane() { return buf.data(); }
  uint8_t* wplane() { return buf.data() + count() * value_bytes(); }

  /* TSDF value as the shaders see it after vs(): float(int16) * (1/32766) for RG16I. */
  inline double F(size_t i) const {
    switch (storage) {
      case KF_STORAGE_F32F32: { float f; std::memcpy(&f, fplane() + 4 * i, 4); return f; }
      case KF_STORAGE_F16U16: { uint16_t h; std::memcpy(&h, fplane() + 2 * i, 2); return half_to_double(h); }
      default: { int16_t q; std::memcpy(&q, fplane() + 2 * i, 2); return (double)q * kShortToF; }
    }
  }
  /* Value used by marching cubes (getVolumeData, histoPyramids.cs:95-107) and summed by
   * the raycast trilinear: the raw int16 for RG16I (scaled afterwards), F otherwise. */
  inline double raw(size_t i) const {
    if (storage == KF_STORAGE_RG16I) { int16_t q; std::memcpy(&q, fplane() + 2 * i, 2); return (double)q; }
    return F(i);
  }
  inline double W(size_t i) const {
    switch (storage) {
      case KF_STORAGE_F32F32: { float f; std::memcpy(&f, wplane() + 4 * i, 4); return f; }
      case KF_STORAGE_F16U16: { uint16_t h; std::memcpy(&h, wplane() + 2 * i, 2); return (double)h; }
      default: { int16_t q; std::memcpy(&q, wplane() + 2 * i, 2); return (double)q; }
    }
  }
  /* set() of integrate.cs:45-50: int(F*32766), int(w) for RG16I. */
  inline void set(size_t i, double f, double w) {
    switch (storage) {
      case KF_STORAGE_F32F32: {
        float ff = (float)f, fw = (float)w;
        std::memcpy(fplane() + 4 * i, &ff, 4);
        std::memcpy(wplane() + 4 * i, &fw, 4);
        break;
      }
      case KF_STORAGE_F16U16: {
        uint16_t lo = half_from_double(f);
        uint16_t hi = (uint16_t)std::min(std::max(w, 0.0), 65535.0);
        std::memcpy(fplane() + 2 * i, &lo, 2);
        std::memcpy(wplane() + 2 * i, &hi, 2);
        break;
      }
      default: {
        int16_t q = (int16_t)(int)(f * 32766.0);
        int16_t qw = (int16_t)(int)w;
        std::memcpy(fplane() + 2 * i, &q, 2);
        std::memcpy(wplane() + 2 * i, &qw, 2);
      }
    }
  }
};

struct PoseEntry {
  double pose[16];
  std::vector<float> depth;
};

struct Level {
  int w = 0, h = 0;
  double fx = 0, fy = 0, cx = 0, cy = 0;
  std::vector<double> depth;  /* mm */
  std::vector<double> vertex; /* 4 per px, camera frame, metres */
  std::vector<double> normal; /* 4 per px */
  std::vector<int32_t> status;
};

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* Accumulate one 6-vector J with residual e and weight h into the 32-float row layout of
 * reduce.cs:226-263 / reduceSDF.cs:52-89. */
inline void accumulate_row(double* s, const double* J, double e, double h, double e2_factor) {
  s[0] += e2_factor * e * e;
  for (int i = 0; i < 6; ++i) s[1 + i] += h * J[i] * e;
  int k = 7;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) s[k++] += h * J[i] * J[j];
}

/* makeJTJ (gFusion.h:472-487): symmetric 6x6 from the 21 upper-triangular sums. */
void make_jtj(const double* v21, double* C) {
  int k = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) { C[i * 6 + j] = v21[k]; C[j * 6 + i] = v21[k]; ++k; }
}

}  // namespace

/* ====================================================================================== */
extern "C" {

void or_euler_xyz(const double a[3], double R[9]) {
  /* glm::eulerAngleXYZ(t1,t2,t3) = Rx(t1) * Ry(t2) * Rz(t3) (glm/gtx/euler_angles),
   * used at gFusion.cpp:700.  Written from the definition; column-major 3x3. */
  double c1 = std::cos(a[0]), s1 = std::sin(a[0]);
  double c2 = std::cos(a[1]), s2 = std::sin(a[1]);
  double c3 = std::cos(a[2]), s3 = std::sin(a[2]);
  double Rx[9] = {1, 0, 0, 0, c1, s1, 0, -s1, c1};
  double Ry[9] = {c2, 0, -s2, 0, 1, 0, s2, 0, c2};
  double Rz[9] = {c3, s3, 0, -s3, c3, 0, 0, 0, 1};
  double T[9];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += Rx[k * 3 + r] * Ry[c * 3 + k];
      T[c * 3 + r] = s;
    }
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += T[k * 3 + r] * Rz[c * 3 + k];
      R[c * 3 + r] = s;
    }
}

void or_se3_exp(const double xi[6], double T[16]) {
  /* exp of Twist(xi) (gFusion.cpp:811-833, .exp() at :866/:996): the 4x4 matrix
   * exponential of [[w]x v; 0 0] in closed form (Rodrigues rotation, V for translation). */
  const double w[3] = {xi[0], xi[1], xi[2]}, v[3] = {xi[3], xi[4], xi[5]};
  double th2 = dot3(w, w), th = std::sqrt(th2);
  double A, B, C;
  if (th < 1e-6) {
    A = 1 - th2 / 6 + th2 * th2 / 120;
    B = 0.5 - th2 / 24 + th2 * th2 / 720;
    C = 1.0 / 6 - th2 / 120 + th2 * th2 / 5040;
  } else {
    A = std::sin(th) / th;
    B = (1 - std::cos(th)) / th2;
    C = (th - std::sin(th)) / (th2 * th);
  }
  double W[9] = {0, w[2], -w[1], -w[2], 0, w[0], w[1], -w[0], 0}; /* col-major [w]x */
  double W2[9];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += W[k * 3 + r] * W[c * 3 + k];
      W2[c * 3 + r] = s;
    }
  double R[9], V[9];
  for (int i = 0; i < 9; ++i) {
    double I = (i % 4 == 0) ? 1.0 : 0.0;
    R[i] = I + A * W[i] + B * W2[i];
    V[i] = I + B * W[i] + C * W2[i];
  }
  std::memset(T, 0, 16 * sizeof(double));
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) T[c * 4 + r] = R[c * 3 + r];
  for (int r = 0; r < 3; ++r) T[12 + r] = V[r] * v[0] + V[3 + r] * v[1] + V[6 + r] * v[2];
  T[15] = 1;
}

/* Symmetric eigen-decomposition by cyclic Jacobi rotations: A (row-major, symmetric) is
 * diagonalised in place, V receives the eigenvectors in its columns. */
static void jacobi_eigen_sym6(double A[36], double V[36]) {
  for (int i = 0; i < 36; ++i) V[i] = (i % 7 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0;
    for (int p = 0; p < 6; ++p)
      for (int q = p + 1; q < 6; ++q) off += A[p * 6 + q] * A[p * 6 + q];
    if (off < 1e-300) break;
    for (int p = 0; p < 6; ++p)
      for (int q = p + 1; q < 6; ++q) {
        double apq = A[p * 6 + q];
        if (std::fabs(apq) < 1e-300) continue;
        double theta = (A[q * 6 + q] - A[p * 6 + p]) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(t * t + 1), sn = t * c;
        for (int k = 0; k < 6; ++k) {
          double akp = A[k * 6 + p], akq = A[k * 6 + q];
          A[k * 6 + p] = c * akp - sn * akq;
          A[k * 6 + q] = sn * akp + c * akq;
        }
        for (int k = 0; k < 6; ++k) {
          double apk = A[p * 6 + k], aqk = A[q * 6 + k];
          A[p * 6 + k] = c * apk - sn * aqk;
          A[q * 6 + k] = sn * apk + c * aqk;
        }
        for (int k = 0; k < 6; ++k) {
          double vkp = V[k * 6 + p], vkq = V[k * 6 + q];
          V[k * 6 + p] = c * vkp - sn * vkq;
          V[k * 6 + q] = sn * vkp + c * vkq;
        }
      }
  }
}

/* The ICP step with the rank guard (Q22; the build's deliberate rule, applied identically
 * by the CUDA path): the minimum-norm least-squares solution that JacobiSVD::solve returns
 * (gFusion.cpp:696-697), x = sum v_i (v_i . b) / l_i over the eigen-directions of C, with
 * the rank cut at tau = 1e-5 of the largest eigenvalue instead of JacobiSVD's 6 * epsilon
 * (which rounding noise of the sums passes).  For a full-rank system this is C^-1 b; for a
 * view of one plane the three unobservable directions get no motion.  Returns the number
 * of directions kept. */
int or_solve_icp_guarded6(const double C[36], const double b[6], double x[6]) {
  const double tau = 1e-5;
  double A[36], V[36];
  std::memcpy(A, C, sizeof(A));
  jacobi_eigen_sym6(A, V);
  double lmax = 0;
  for (int k = 0; k < 6; ++k) lmax = std::max(lmax, A[k * 7]);
  for (int i = 0; i < 6; ++i) x[i] = 0;
  int kept = 0;
  for (int k = 0; k < 6; ++k) {
    double l = A[k * 7];
    if (!(l > 0 && l >= tau * lmax)) continue;
    ++kept;
    double vb = 0;
    for (int i = 0; i < 6; ++i) vb += V[i * 6 + k] * b[i];
    for (int i = 0; i < 6; ++i) x[i] += V[i * 6 + k] * vb / l;
  }
  return kept;
}

int or_solve_pinv6(const double Cin[36], const double b[6], double x[6]) {
  /* Symmetric Jacobi eigen-decomposition; x = sum_i (u_i.b / l_i) u_i over eigenvalues
   * above 6*eps*max|l| — the minimum-norm least-squares solution JacobiSVD::solve
   * returns (gFusion.cpp:696-697). */
  double A[36], V[36];
  std::memcpy(A, Cin, sizeof(A));
  for (int i = 0; i < 36; ++i) V[i] = (i % 7 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0;
    for (int p = 0; p < 6; ++p)
      for (int q = p + 1; q < 6; ++q) off += A[p * 6 + q] * A[p * 6 + q];
    if (off < 1e-300) break;
    for (int p = 0; p < 6; ++p)
      for (int q = p + 1; q < 6; ++q) {
        double apq = A[p * 6 + q];
        if (std::fabs(apq) < 1e-300) continue;
        double theta = (A[q * 6 + q] - A[p * 6 + p]) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 6; ++k) {
          double akp = A[k * 6 + p], akq = A[k * 6 + q];
          A[k * 6 + p] = c * akp - s * akq;
          A[k * 6 + q] = s * akp + c * akq;
        }
        for (int k = 0; k < 6; ++k) {
          double apk = A[p * 6 + k], aqk = A[q * 6 + k];
          A[p * 6 + k] = c * apk - s * aqk;
          A[q * 6 + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 6; ++k) {
          double vkp = V[k * 6 + p], vkq = V[k * 6 + q];
          V[k * 6 + p] = c * vkp - s * vkq;
          V[k * 6 + q] = s * vkp + c * vkq;
        }
      }
  }
  double lmax = 0;
  for (int i = 0; i < 6; ++i) lmax = std::max(lmax, std::fabs(A[i * 6 + i]));
  double thr = 6 * 2.220446049250313e-16 * lmax;
  for (int i = 0; i < 6; ++i) x[i] = 0;
  int rank = 0;
  for (int i = 0; i < 6; ++i) {
    double l = A[i * 6 + i];
    if (!(std::fabs(l) > thr)) continue;
    ++rank;
    double ub = 0;
    for (int k = 0; k < 6; ++k) ub += V[k * 6 + i] * b[k];
    for (int k = 0; k < 6; ++k) x[k] += V[k * 6 + i] * ub / l;
  }
  return rank;
}

int or_solve_ldlt6(const double C[36], const double b[6], double x[6]) {
  /* C.ldlt().solve(b) (gFusion.cpp:902) for the symmetric damped system; unpivoted LDL^T
   * (identical solution for SPD C; NaN in, NaN out). */
  double L[36] = {0}, D[6];
  for (int j = 0; j < 6; ++j) {
    double d = C[j * 6 + j];
    for (int k = 0; k < j; ++k) d -= L[j * 6 + k] * L[j * 6 + k] * D[k];
    D[j] = d;
    L[j * 6 + j] = 1;
    for (int i = j + 1; i < 6; ++i) {
      double v = C[i * 6 + j];
      for (int k = 0; k < j; ++k) v -= L[i * 6 + k] * L[j * 6 + k] * D[k];
      L[i * 6 + j] = v / d;
    }
  }
  double y[6];
  for (int i = 0; i < 6; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= L[i * 6 + k] * y[k];
    y[i] = v;
  }
  for (int i = 0; i < 6; ++i) y[i] /= D[i];
  for (int i = 5; i >= 0; --i) {
    double v = y[i];
    for (int k = i + 1; k < 6; ++k) v -= L[k * 6 + i] * x[k];
    x[i] = v;
  }
  return 0;
}

int or_mc_tables(uint16_t edge[256], int8_t tri[256 * 16], uint8_t nverts[256],
                 uint8_t ntri[256], uint8_t offsets3[72]) {
  std::memcpy(edge, kf_mc_edge_table, sizeof(kf_mc_edge_table));
  std::memcpy(tri, kf_mc_tri_table, sizeof(kf_mc_tri_table));
  std::memcpy(nverts, kf_mc_num_verts, sizeof(kf_mc_num_verts));
  std::memcpy(ntri, kf_mc_nr_triangles, sizeof(kf_mc_nr_triangles));
  std::memcpy(offsets3, kf_mc_offsets3, sizeof(kf_mc_offsets3));
  return KF_OK;
}

int or_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#endif
  return KF_OK;
}

int or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int or_prefix_sum_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total) {
  /* Exclusive scan of prefixSum.cs:28-197 with the total of mcubes.cpp:196-203
   * (lastElement + lastScanElement); unsigned 32-bit wrap-around like GLSL uint. */
  uint32_t acc = 0;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t v = in[i];
    out[i] = acc;
    acc += v;
  }
  if (total) *total = acc;
  return KF_OK;
}

}  // extern "C"

/* ====================================================================================== */
struct or_session {
  kf_config cfg;
  kf_intrinsics intr;
  Volume vol;
  Level lv[3];
  double pose[16];
  double pose_eig[16];
  double raycast_pose[16]; /* pose of the last raycast (clean Q4 association) */
  double cum_twist[6] = {0, 0, 0, 0, 0, 0};
  std::vector<PoseEntry> library;
  std::vector<double> ref_vertex, ref_normal; /* raycast output, 4 per px */
  std::vector<double> sdf_rows;               /* persistent trackSDF SSBO, 8 per px */
  double last_sums[32];
  double ae = 0;
  int counter = 0;
  bool reset_window = true;
  /* depth ingest before the pyramid (libfreenect2 undistortion, filter3D.cs) */
  bool undistort = false;
  bool depth_filter = false;
  std::vector<int32_t> undistort_map;
  /* marching cubes */
  std::vector<uint32_t> mc_base;                /* nx*ny*nz, numTri | ci << 16 */
  std::vector<std::vector<uint32_t>> mc_levels; /* level k>=1, (P>>k)^3 */
  std::vector<float> mc_vertices;               /* 4 per vertex */
  std::vector<float> mc_normals;                /* 4 per vertex: the face normal, w = 0 */
  std::vector<float> mesh_pos, mesh_nrm;        /* welded mesh: 3 per vertex */
  std::vector<uint32_t> mesh_idx;               /* 3 per triangle */
  int mesh_valid = 0;
  uint32_t mc_triangles = 0;
  int mc_valid = 0;
};

namespace {

void level_setup(or_session* s) {
  for (int l = 0; l < 3; ++l) {
    Level& L = s->lv[l];
    L.w = s->intr.width >> l;
    L.h = s->intr.height >> l;
    double sc = (double)(1 << l);
    /* m_camPamsDepth / float(1 << i) (gFusion.cpp:517) */
    L.fx = s->intr.fx / sc; L.fy = s->intr.fy / sc;
    L.cx = s->intr.cx / sc; L.cy = s->intr.cy / sc;
    size_t n = (size_t)L.w * L.h;
    L.depth.assign(n, 0.0);
    L.vertex.assign(4 * n, 0.0);
    L.normal.assign(4 * n, 0.0);
    L.status.assign(n, 0);
  }
  size_t n0 = (size_t)s->intr.width * s->intr.height;
  s->ref_vertex.assign(4 * n0, 0.0);
  s->ref_normal.assign(4 * n0, 0.0);
  s->sdf_rows.assign(8 * n0, 0.0);
}

/* ---- depth ingest: Kinect-v2 undistortion (libfreenect2) and filter3D.cs ------------------
 * The reference feeds the fusion with libfreenect2's `undistorted` depth frame
 * (src/interface.cpp:290-313, Registration::apply; the library is philipNoonan/libfreenect2
 * at commit 0ee1ee2f8d2331253e78aaac0a340436b14ba34e, depends/libfreenect2-nm/portfile.cmake,
 * not part of the reference tree).  Registration's published algorithm: for every
 * undistorted pixel (x, y), distort() applies the IR camera's Brown-Conrady model (radial
 * k1, k2, k3; tangential p1, p2) in float, the source pixel is (int)(m + 0.5f) on each axis,
 * and pixels whose source falls outside the image get depth 0; apply() copies the raw depth
 * through that map.  This restatement evaluates the same float expressions in the same order
 * (no fused multiply-adds: the oracle is built for x86-64-v2, which has none). */
#if defined(__FMA__)
#error "the undistortion map is specified without fused multiply-adds; build for a target without FMA"
#endif
int32_t undistort_index(const float ir[9], int x, int y, int W, int H) {
  const float fx = ir[0], fy = ir[1], cx = ir[2], cy = ir[3];
  const float k1 = ir[4], k2 = ir[5], k3 = ir[6], p1 = ir[7], p2 = ir[8];
  const float dx = ((float)x - cx) / fx;
  const float dy = ((float)y - cy) / fy;
  const float dx2 = dx * dx, dy2 = dy * dy;
  const float r2 = dx2 + dy2;
  const float dxdy2 = 2 * dx * dy;
  const float kr = 1 + ((k3 * r2 + k2) * r2 + k1) * r2;
  const float mx = fx * (dx * kr + p2 * (r2 + 2 * dx2) + p1 * dxdy2) + cx;
  const float my = fy * (dy * kr + p1 * (r2 + 2 * dy2) + p2 * dxdy2) + cy;
  const float vx = mx + 0.5f, vy = my + 0.5f;
  /* (int) truncates towards zero: a source index is inside the image iff v > -1 and v < size */
  if (!(vx > -1.0f && vx < (float)W && vy > -1.0f && vy < (float)H)) return -1;
  return (int32_t)vy * W + (int32_t)vx;
}

/* filter3D.cs:23-86: a depth is valid when 5 < d < 4000 (checkPixel); an interior pixel
 * (1 < x < W-1, 1 < y < H-1) keeps its depth when more than 6 of its 3x3 neighbourhood are
 * valid and it lies within 5 mm of their mean, else 0.  Float arithmetic, neighbourhood
 * summed column by column (the shader's i (x) outer, j (y) inner loops).  The shader never
 * writes the border pixels (its dispatch offset pix.y += 2 only moves rows inside that
 * rule); they are 0 here. */
inline float check_pixel(float v) { return (v > 5.0f && v < 4000.0f) ? v : 0.0f; }

void filter3d(const float* in, float* out, int W, int H) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      float o = 0.0f;
      if (x > 1 && x < W - 1 && y > 1 && y < H - 1) {
        float valid = 9.0f, sum = 0.0f, curr = 0.0f;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            const float t = check_pixel(in[(size_t)(y + j - 1) * W + (x + i - 1)]);
            if (t == 0.0f) valid -= 1.0f;
            else sum += t;
            if (i == 1 && j == 1) curr = t;
          }
        const float mean = valid > 6.0f ? sum / valid : 0.0f;
        if (mean > 0.0f && std::fabs(curr - mean) < 5.0f) o = curr;
      }
      out[(size_t)y * W + x] = o;
    }
}

/* The level-0 depth the pyramid is built from: raw input, undistorted, then filtered. */
void prepare_depth(or_session* s, const float* raw) {
  Level& L = s->lv[0];
  const int W = L.w, H = L.h;
  const size_t n = (size_t)W * H;
  std::vector<float> a(raw, raw + n), b(n);
  if (s->undistort) {
    for (size_t i = 0; i < n; ++i) b[i] = s->undistort_map[i] < 0 ? 0.0f : a[(size_t)s->undistort_map[i]];
    a.swap(b);
  }
  if (s->depth_filter) {
    filter3d(a.data(), b.data(), W, H);
    a.swap(b);
  }
  for (size_t i = 0; i < n; ++i) L.depth[i] = a[i];
}

/* ---- depthToVertex: mip + depthToVert.cs:33-72 ---------------------------------------- */
void depth_to_vertex(or_session* s) {
  for (int l = 1; l < 3; ++l) {
    /* glGenerateMipmap (gFusion.cpp:508): 2x2 box mean of the previous level, zeros
     * included. */
    Level& P = s->lv[l - 1];
    Level& L = s->lv[l];
#pragma omp parallel for schedule(static)
    for (int y = 0; y < L.h; ++y)
      for (int x = 0; x < L.w; ++x) {
        const double* p = &P.depth[(size_t)(2 * y) * P.w + 2 * x];
        L.depth[(size_t)y * L.w + x] = 0.25 * ((p[0] + p[1]) + (p[P.w] + p[P.w + 1]));
      }
  }
  for (int l = 0; l < 3; ++l) {
    Level& L = s->lv[l];
    double ifx = 1.0 / L.fx, ify = 1.0 / L.fy;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < L.h; ++y)
      for (int x = 0; x < L.w; ++x) {
        size_t i = (size_t)y * L.w + x;
        double d = L.depth[i] / 1000.0;
        /* (depth/1000) * rotate(invK, (u, v, 1)) with invK from getInverseCameraMatrix */
        double* v = &L.vertex[4 * i];
        v[0] = d * (x * ifx - L.cx * ifx);
        v[1] = d * (y * ify - L.cy * ify);
        v[2] = d;
        v[3] = 0;
      }
  }
}

/* ---- vertexToNormal: vertToNorm.cs:9-57 ----------------------------------------------- */
void vertex_to_normal(or_session* s) {
  const bool q3 = s->cfg.quirks & KF_Q3_DOWN_FROM_LEFT;
  for (int l = 0; l < 3; ++l) {
    Level& L = s->lv[l];
    auto load = [&](long x, long y, double* out) {
      /* imageLoad returns 0 out of bounds; pix.x - 1 at x == 0 wraps as uint -> -1 */
      if (x < 0 || y < 0 || x >= L.w || y >= L.h) { out[0] = out[1] = out[2] = 0; return; }
      const double* v = &L.vertex[4 * ((size_t)y * L.w + x)];
      out[0] = v[0]; out[1] = v[1]; out[2] = v[2];
    };
#pragma omp parallel for schedule(static)
    for (int y = 0; y < L.h; ++y)
      for (int x = 0; x < L.w; ++x) {
        double lf[3], rt[3], up[3], dn[3];
        load(x - 1, y, lf);                               /* max(pix.x-1,0) on uint */
        load(std::min(x + 1, L.w - 1), y, rt);
        load(x, y - 1, up);
        load(q3 ? x - 1 : x, std::min(y + 1, L.h - 1), dn); /* Q3: column x-1 */
        double* n = &L.normal[4 * ((size_t)y * L.w + x)];
        if (lf[2] == 0 || rt[2] == 0 || up[2] == 0 || dn[2] == 0) {
          n[0] = 2; n[1] = 0; n[2] = 0; n[3] = 0;
        } else {
          double dx[3] = {rt[0] - lf[0], rt[1] - lf[1], rt[2] - lf[2]};
          double dy[3] = {dn[0] - up[0], dn[1] - up[1], dn[2] - up[2]};
          double c[3];
          cross3(dy, dx, c);
          double len = std::sqrt(dot3(c, c));
          n[0] = c[0] / len; n[1] = c[1] / len; n[2] = c[2] / len; n[3] = 1;
        }
      }
  }
}

/* ---- track.cs:47-163 + reduce.cs:27-126 for one ICP iteration ------------------------- */
void icp_track_reduce(or_session* s, int level, double* sums) {
  Level& L = s->lv[level];
  const int W0 = s->intr.width, H0 = s->intr.height;
  double K[16], invT[16], view[16];
  camera_matrix(s->intr.fx, s->intr.fy, s->intr.cx, s->intr.cy, K); /* level-0 K, :747 */
  /* Q4: K * inverse(m_pose) with the current estimate; clean: the raycast pose */
  mat4_inverse((s->cfg.quirks & KF_Q4_SAME_PIXEL) ? s->pose : s->raycast_pose, invT);
  mat4_mul(K, invT, view); /* projectReference = K * inverse(m_pose) (gFusion.cpp:747) */
  const double* T = s->pose;
  const double dist = s->cfg.dist_threshold, nthr = s->cfg.normal_threshold;
  const bool q1 = s->cfg.quirks & KF_Q1_LAST_GROUP_ONLY;
  std::vector<double> rows((size_t)L.h * 32, 0.0);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < L.h; ++y) {
    double* acc = &rows[(size_t)y * 32];
    for (int x = 0; x < L.w; ++x) {
      size_t i = (size_t)y * L.w + x;
      const double* n = &L.normal[4 * i];
      const double* v = &L.vertex[4 * i];
      int status;
      double e = 0, J[6] = {0, 0, 0, 0, 0, 0};
      if (n[0] == 2) {
        status = -1;
      } else if (v[2] == 0) {
        /* z == 0 with a valid normal projects (0,0,0): 0/0 in track.cs:72, undefined in
         * GLSL.  Guarded as "outside the image". */
        status = -2;
      } else {
        double pv[3], pp[3];
        xform(T, v, 1.0, pv);     /* Ttrack * vec4(v, 1) */
        xform(view, pv, 1.0, pp); /* view * projectedVertex */
        double px = pp[0] / pp[2] + 0.5, py = pp[1] / pp[2] + 0.5;
        if (!(px >= 0) || px > W0 - 1 || !(py >= 0) || py > H0 - 1) {
          status = -2;
        } else {
          int rx = (int)px, ry = (int)py;
          size_t ri = (size_t)ry * W0 + rx;
          const double* rn = &s->ref_normal[4 * ri];
          const double* rv = &s->ref_vertex[4 * ri];
          if (rn[0] == -2) {
            status = -3;
          } else {
            double diff[3] = {rv[0] - pv[0], rv[1] - pv[1], rv[2] - pv[2]};
            double pn[3];
            xform(T, n, 0.0, pn); /* rotate(Ttrack, normal) */
            if (std::sqrt(dot3(diff, diff)) > dist) {
              status = -4;
            } else if (dot3(pn, rn) < nthr) {
              status = -5;
            } else {
              status = 1;
              e = dot3(rn, diff);
              J[0] = rn[0]; J[1] = rn[1]; J[2] = rn[2];
              cross3(pv, rn, &J[3]);
            }
          }
        }
      }
      L.status[i] = status;
      if (q1 && (y % 8) != 7) continue;
      /* reduce.cs:209-263: every pixel adds to the count, valid ones to the sums */
      acc[28] += 1;
      if (status < 1) continue;
      accumulate_row(acc, J, e, 1.0, 1.0);
    }
  }
  std::fill(sums, sums + 32, 0.0);
  for (int y = 0; y < L.h; ++y)
    for (int k = 0; k < 32; ++k) sums[k] += rows[(size_t)y * 32 + k];
}

void update_pose_finder(or_session* s);

/* ---- Track(): gFusion.cpp:648-740 ------------------------------------------------------ */
bool track_icp(or_session* s) {
  double old_pose[16];
  std::memcpy(old_pose, s->pose, sizeof(old_pose));
  double ae = 0;
  for (int level = 2; level >= 0; --level) {
    for (int it = 0; it < s->cfg.iterations[level]; ++it) {
      double sums[32];
      icp_track_reduce(s, level, sums);
      std::memcpy(s->last_sums, sums, sizeof(sums));
      double b[6], C[36];
      for (int i = 0; i < 6; ++i) b[i] = sums[1 + i];
      make_jtj(&sums[7], C);
      ae = std::sqrt(sums[0] / sums[28]); /* getReduction :1167 */
      double x[6];
      or_solve_icp_guarded6(C, b, x); /* JacobiSVD::solve with the rank guard (Q22) */
      /* delta = eulerAngleXYZ(x3,x4,x5); delta[3].xyz = x0..2; m_pose = delta * m_pose */
      double R[9], delta[16];
      or_euler_xyz(&x[3], R);
      std::memset(delta, 0, sizeof(delta));
      for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) delta[c * 4 + r] = R[c * 3 + r];
      delta[12] = x[0]; delta[13] = x[1]; delta[14] = x[2]; delta[15] = 1;
      mat4_mul(delta, s->pose, s->pose);
      double nrm = 0;
      for (int i = 0; i < 6; ++i) nrm += x[i] * x[i];
      nrm = std::sqrt(nrm);
      if (nrm < 1e-5 && nrm != 0) break;
    }
  }
  s->ae = ae;
  if (ae > 0.5 || ae == 0) {
    std::memcpy(s->pose, old_pose, sizeof(old_pose));
    return false;
  }
  update_pose_finder(s);
  return true;
}

/* ---- SDF sampling of trackSDF.cs:193-237 ----------------------------------------------- */
inline double vol_tap(const Volume& V, long x, long y, long z) {
  if (x < 0 || y < 0 || z < 0 || x >= V.nx || y >= V.ny || z >= V.nz) return 0.0;
  return V.F(V.idx((int)x, (int)y, (int)z));
}

double sdf_sample(const Volume& V, const double* loc) {
  double fi = std::trunc(loc[0]), fj = std::trunc(loc[1]), fk = std::trunc(loc[2]);
  double x = loc[0] - fi, y = loc[1] - fj, z = loc[2] - fk; /* modf */
  long I = (long)fi, J = (long)fj, Kk = (long)fk;
  double N0 = vol_tap(V, I, J, Kk), N1 = vol_tap(V, I, J + 1, Kk);
  double N2 = vol_tap(V, I + 1, J, Kk), N3 = vol_tap(V, I + 1, J + 1, Kk);
  double N4 = vol_tap(V, I, J, Kk + 1), N5 = vol_tap(V, I, J + 1, Kk + 1);
  double N6 = vol_tap(V, I + 1, J, Kk + 1), N7 = vol_tap(V, I + 1, J + 1, Kk + 1);
  double a0 = N0 * (1.0 - z) + N4 * z, a1 = N1 * (1.0 - z) + N5 * z;
  double b0 = N2 * (1.0 - z) + N6 * z, b1 = N3 * (1.0 - z) + N7 * z;
  return (a0 * (1.0 - y) + a1 * y) * (1.0 - x) + (b0 * (1.0 - y) + b1 * y) * x;
}

/* ---- trackSDF.cs:407-531 + reduceSDF.cs:28-116 ---------------------------------------- */
void sdf_track_reduce(or_session* s, int level, const double* T, double* sums) {
  Level& L = s->lv[level];
  const Volume& V = s->vol;
  const bool q1 = s->cfg.quirks & KF_Q1_LAST_GROUP_ONLY;
  const bool q6 = s->cfg.quirks & KF_Q6_SDF_D2_TWICE;
  const bool q7 = s->cfg.quirks & KF_Q7_SDF_LAST_COLUMN;
  const bool q23 = s->cfg.quirks & KF_Q23_SDF_XY_OFFSET;
  const double sx = V.nx / s->cfg.dim_x, sy = V.ny / s->cfg.dim_y, sz = V.nz / s->cfg.dim_z;
  const double vsz = s->cfg.dim_x / V.nx; /* volDim.x / volSize.x for every axis, :235 */
  const int xend = q7 ? L.w - 1 : L.w;
  std::vector<double> rows((size_t)L.h * 32, 0.0);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < L.h; ++y) {
    for (int x = 0; x < xend; ++x) {
      size_t i = (size_t)y * L.w + x;
      const double* cp = &L.vertex[4 * i];
      double p[3];
      xform(T, cp, 1.0, p);
      double cvp[3];
      if (q23) { /* vec3(a - 0.5, b - 0.5, c) - 0.5 (trackSDF.cs:429) */
        cvp[0] = p[0] * sx - 0.5 - 0.5;
        cvp[1] = p[1] * sy - 0.5 - 0.5;
        cvp[2] = p[2] * sz - 0.5;
      } else {
        cvp[0] = p[0] * sx - 0.5;
        cvp[1] = p[1] * sy - 0.5;
        cvp[2] = p[2] * sz - 0.5;
      }
      double D = sdf_sample(V, cvp);
      double g[3];
      for (int a = 0; a < 3; ++a) {
        double up[3] = {cvp[0], cvp[1], cvp[2]}, dn[3] = {cvp[0], cvp[1], cvp[2]};
        up[a] += 1.0;
        dn[a] -= 1.0;
        g[a] = (sdf_sample(V, up) - sdf_sample(V, dn)) / (2.0 * vsz);
      }
      double* row = &s->sdf_rows[8 * i];
      if (D < 1.0 && D > -1.0) {
        double J[6];
        cross3(p, g, J); /* dsdf . dx/dxi with dx/dxi = [[p]x^T | I], :459-468 */
        J[3] = g[0]; J[4] = g[1]; J[5] = g[2];
        double ad = std::fabs(D);
        double h = ad < 0.02 ? 1.0 : 0.02 / ad;
        row[0] = h; row[1] = D;
        for (int k = 0; k < 6; ++k) row[2 + k] = J[k];
      } else {
        for (int k = 0; k < 8; ++k) row[k] = 0;
      }
    }
  }
  /* reduceSDF over the full level image, reading the persistent rows (Q7: the last
   * column holds whatever an earlier call left there) */
#pragma omp parallel for schedule(static)
  for (int y = 0; y < L.h; ++y) {
    double* acc = &rows[(size_t)y * 32];
    if (q1 && (y % 8) != 7) continue;
    for (int x = 0; x < L.w; ++x) {
      const double* row = &s->sdf_rows[8 * ((size_t)y * L.w + x)];
      accumulate_row(acc, &row[2], row[1], row[0], q6 ? 2.0 : 1.0);
      acc[28] += 1;
    }
  }
  std::fill(sums, sums + 32, 0.0);
  for (int y = 0; y < L.h; ++y)
    for (int k = 0; k < 32; ++k) sums[k] += rows[(size_t)y * 32 + k];
}

/* ---- TrackSDF(): gFusion.cpp:835-1038 --------------------------------------------------- */
bool track_sdf(or_session* s) {
  bool tracked = false;
  double old_pose[16], prev[16];
  std::memcpy(old_pose, s->pose, sizeof(old_pose));
  std::memcpy(prev, s->pose_eig, sizeof(prev));
  double result[6] = {0, 0, 0, 0, 0, 0}, result_prev[6] = {0, 0, 0, 0, 0, 0};
  double ae = 0;
  for (int level = 2; level >= 0; --level) {
    for (int it = 0; it < s->cfg.iterations[level]; ++it) {
      double E[16], T[16];
      or_se3_exp(result, E);
      mat4_mul(E, prev, T); /* camToWorld = exp(Twist(result)) * m_pose_eig_prev */
      double sums[32];
      sdf_track_reduce(s, level, T, sums);
      std::memcpy(s->last_sums, sums, sizeof(sums));
      double b[6], C[36];
      for (int i = 0; i < 6; ++i) b[i] = sums[1 + i];
      make_jtj(&sums[7], C);
      ae = std::sqrt(sums[0] / sums[28]);
      double mx = C[0];
      for (int i = 1; i < 36; ++i) mx = std::max(mx, C[i]); /* maxCoeff, :890 */
      double scaling = 1.0 / mx;
      for (int i = 0; i < 36; ++i) C[i] *= scaling;
      for (int i = 0; i < 6; ++i) b[i] *= scaling;
      for (int i = 0; i < 6; ++i) C[i * 7] += (double)it * 0.01;
      double dx[6];
      or_solve_ldlt6(C, b, dx);
      double cn = 0;
      for (int i = 0; i < 6; ++i) {
        result[i] -= dx[i];
        double ch = result[i] - result_prev[i];
        cn += ch * ch;
        result_prev[i] = result[i];
      }
      cn = std::sqrt(cn);
      if ((ae != 0 && ae < 1e-3) || cn < 1e-3) {
        tracked = true;
        break; /* inner loop only (:906-920) */
      }
    }
  }
  s->ae = ae;
  double sum = 0;
  for (int i = 0; i < 6; ++i) sum += result[i];
  if (std::isnan(sum))
    for (int i = 0; i < 6; ++i) result[i] = 0;
  if (tracked) {
    double E[16];
    or_se3_exp(result, E);
    mat4_mul(E, prev, s->pose_eig);
    std::memcpy(s->pose, s->pose_eig, sizeof(s->pose));
    for (int i = 0; i < 6; ++i) s->cum_twist[i] += result[i];
  } else {
    std::memcpy(s->pose_eig, prev, sizeof(prev));
    std::memcpy(s->pose, old_pose, sizeof(old_pose));
  }
  return tracked;
}

/* ---- updatePoseFinder / addPoseToLibrary (gFusion.cpp:1570-1614) ------------------------ */
void update_pose_finder(or_session* s) {
  for (const PoseEntry& e : s->library) {
    double dx = e.pose[12] - s->pose[12], dy = e.pose[13] - s->pose[13],
           dz = e.pose[14] - s->pose[14];
    if (std::sqrt(dx * dx + dy * dy + dz * dz) < 0.2) return;
  }
  PoseEntry e;
  std::memcpy(e.pose, s->pose, sizeof(e.pose));
  e.depth.resize(s->lv[0].depth.size());
  for (size_t i = 0; i < e.depth.size(); ++i) e.depth[i] = (float)s->lv[0].depth[i];
  s->library.push_back(std::move(e));
}

/* ---- recoverPose (gFusion.cpp:1616-1653) ----------------------------------------------- */
bool recover_pose(or_session* s) {
  if (s->library.empty()) return false;
  for (const PoseEntry& e : s->library) {
    std::memcpy(s->pose, e.pose, sizeof(s->pose));
    if (track_sdf(s)) return true;
  }
  return false;
}

/* ---- integrate.cs:52-169 ----------------------------------------------------------------- */
void integrate(or_session* s) {
  Volume& V = s->vol;
  const Level& L0 = s->lv[0];
  double invT[16];
  mat4_inverse(s->pose, invT); /* glm::inverse(m_pose), gFusion.cpp:1242 */
  const double fx = s->intr.fx, fy = s->intr.fy, cx = s->intr.cx, cy = s->intr.cy;
  const int W = s->intr.width, H = s->intr.height; /* 512x424 hard-coded at :54 (Q11) */
  const double mu = s->cfg.mu, maxw = s->cfg.max_weight;
  const bool band = s->cfg.quirks & KF_Q8_NARROW_BAND;
  const double vx = s->cfg.dim_x / V.nx, vy = s->cfg.dim_y / V.ny, vz = s->cfg.dim_z / V.nz;
  /* delta = rotate(invTrack, (0, 0, volDim.z / volSize.z)) */
  const double dz[3] = {Mc(invT, 2, 0) * vz, Mc(invT, 2, 1) * vz, Mc(invT, 2, 2) * vz};
#pragma omp parallel for collapse(2) schedule(static)
  for (int y = 0; y < V.ny; ++y)
    for (int x = 0; x < V.nx; ++x) {
      double c[3] = {(x + 0.5) * vx, (y + 0.5) * vy, 0.5 * vz};
      double p0[3];
      xform(invT, c, 1.0, p0);
      for (int z = 0; z < V.nz; ++z) {
        double pos[3] = {p0[0] + z * dz[0], p0[1] + z * dz[1], p0[2] + z * dz[2]};
        if (pos[2] < 0.0001) continue;
        double cx3 = fx * pos[0] + cx * pos[2], cy3 = fy * pos[1] + cy * pos[2];
        double px = cx3 / pos[2] + 0.5, py = cy3 / pos[2] + 0.5;
        if (px < 0 || px > W - 1 || py < 0 || py > H - 1) continue;
        int u = (int)px, v = (int)py;
        double d = L0.depth[(size_t)v * W + u] / 1000.0;
        if (d == 0) continue;
        double rx = pos[0] / pos[2], ry = pos[1] / pos[2];
        double diff = (d - pos[2]) * std::sqrt(1.0 + rx * rx + ry * ry);
        size_t vi = V.idx(x, y, z);
        if (diff > -mu) {
          double sdf = std::min(1.0, diff / mu);
          double F = V.F(vi), w = V.W(vi);
          double wd = (w * F + sdf) / (w + 1.0);
          if (!band) {
            /* the reference's earlier update (integrate.cs:115-150) */
            F = std::min(std::max(wd, -1.0), 1.0);
            w = std::min(w + 1.0, maxw);
          } else if (wd < 0.2) {
            F = std::min(std::max(wd, -0.1), 0.2);
            w = std::min(w + 1.0, maxw);
          } else {
            F = 0; w = 0;
          }
          V.set(vi, F, w);
        } else {
          V.set(vi, 0.0, 0.0);
        }
      }
    }
}

/* ---- raycast.cs:69-82 interpVol and :229-276 getGradient -------------------------------- */
struct RaySampler {
  const Volume& V;
  double sx, sy, sz, scale;
  explicit RaySampler(const or_session* s) : V(s->vol) {
    sx = V.nx / s->cfg.dim_x; sy = V.ny / s->cfg.dim_y; sz = V.nz / s->cfg.dim_z;
    scale = (V.storage == KF_STORAGE_RG16I) ? kShortToF : 1.0;
  }
  inline double vs(int x, int y, int z) const { return V.raw(V.idx(x, y, z)); }
  double interp(const double* p) const {
    double q[3] = {p[0] * sx - 0.5, p[1] * sy - 0.5, p[2] * sz - 0.5};
    int n[3] = {V.nx, V.ny, V.nz};
    int lo[3], hi[3];
    double f[3];
    for (int a = 0; a < 3; ++a) {
      double b = std::floor(q[a]);
      f[a] = q[a] - b;
      int bi = (int)b;
      lo[a] = std::min(std::max(bi, 0), n[a] - 1);
      hi[a] = std::min(bi + 1, n[a] - 1);
      hi[a] = std::max(hi[a], 0);
    }
    double v =
        ((vs(lo[0], lo[1], lo[2]) * (1 - f[0]) + vs(hi[0], lo[1], lo[2]) * f[0]) * (1 - f[1]) +
         (vs(lo[0], hi[1], lo[2]) * (1 - f[0]) + vs(hi[0], hi[1], lo[2]) * f[0]) * f[1]) * (1 - f[2]) +
        ((vs(lo[0], lo[1], hi[2]) * (1 - f[0]) + vs(hi[0], lo[1], hi[2]) * f[0]) * (1 - f[1]) +
         (vs(lo[0], hi[1], hi[2]) * (1 - f[0]) + vs(hi[0], hi[1], hi[2]) * f[0]) * f[1]) * f[2];
    return v * scale;
  }
  void gradient(const double* h, double* g) const {
    double q[3] = {h[0] * sx - 0.5, h[1] * sy - 0.5, h[2] * sz - 0.5};
    int n[3] = {V.nx, V.ny, V.nz};
    int ll[3], lu[3], ul[3], uu[3];
    double f[3];
    for (int a = 0; a < 3; ++a) {
      double b = std::floor(q[a]);
      f[a] = q[a] - b;
      int bi = (int)b;
      ll[a] = std::min(std::max(bi - 1, 0), n[a] - 1);
      lu[a] = std::min(std::max(bi, 0), n[a] - 1);
      ul[a] = std::max(std::min(bi + 1, n[a] - 1), 0);
      uu[a] = std::max(std::min(bi + 2, n[a] - 1), 0);
    }
    const int* lo = lu;
    const int* up = ul;
    /* one axis: trilinear of (v(upper_lower) - v(lower_lower)) at the lower corner and
     * (v(upper_upper) - v(lower_upper)) at the upper corner, :243-271 */
    for (int a = 0; a < 3; ++a) {
      double acc = 0;
      for (int cz = 0; cz < 2; ++cz)
        for (int cy = 0; cy < 2; ++cy)
          for (int cxx = 0; cxx < 2; ++cxx) {
            int c[3] = {cxx, cy, cz};
            int pa[3], pb[3];
            for (int k = 0; k < 3; ++k) {
              if (k == a) {
                pa[k] = c[k] ? uu[k] : ul[k];
                pb[k] = c[k] ? lu[k] : ll[k];
              } else {
                pa[k] = c[k] ? up[k] : lo[k];
                pb[k] = pa[k];
              }
            }
            double wgt = (c[0] ? f[0] : 1 - f[0]) * (c[1] ? f[1] : 1 - f[1]) *
                         (c[2] ? f[2] : 1 - f[2]);
            acc += wgt * (vs(pa[0], pa[1], pa[2]) - vs(pb[0], pb[1], pb[2]));
          }
      g[a] = acc;
    }
    /* * volDim/volSize * (0.5 * 1/32766), :273 (Q10: multiplied, not divided) */
    g[0] *= (1.0 / sx) * 0.5 * scale;
    g[1] *= (1.0 / sy) * 0.5 * scale;
    g[2] *= (1.0 / sz) * 0.5 * scale;
  }
};

/* ---- raycast(): gFusion.cpp:1289-1366 + raycast.cs:133-321 -------------------------------- */
void raycast(or_session* s) {
  const int W = s->intr.width, H = s->intr.height;
  double invK[16], view[16];
  std::memset(invK, 0, sizeof(invK));
  M(invK, 0, 0) = 1.0 / s->intr.fx; M(invK, 2, 0) = -s->intr.cx / s->intr.fx;
  M(invK, 1, 1) = 1.0 / s->intr.fy; M(invK, 2, 1) = -s->intr.cy / s->intr.fy;
  M(invK, 2, 2) = 1; M(invK, 3, 3) = 1;
  mat4_mul(s->pose, invK, view); /* view = m_pose * invK */
  std::memcpy(s->raycast_pose, s->pose, sizeof(s->pose));
  const double dim[3] = {s->cfg.dim_x, s->cfg.dim_y, s->cfg.dim_z};
  /* stepSize(): min(volDim) / max(volSize) (gFusion.h:72-81) */
  const double step = std::min(std::min(dim[0], dim[1]), dim[2]) /
                      (double)std::max(std::max(s->vol.nx, s->vol.ny), s->vol.nz);
  const double large_step = 0.75 * s->cfg.mu;
  const double nearp = s->cfg.near_plane, farp = s->cfg.far_plane;
  RaySampler rs(s);
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      double o[3] = {Mc(view, 3, 0), Mc(view, 3, 1), Mc(view, 3, 2)};
      double pix[3] = {(double)x, (double)y, 1.0};
      double d[3];
      xform(view, pix, 0.0, d);
      double tmin[3], tmax[3];
      for (int a = 0; a < 3; ++a) {
        double inv = 1.0 / d[a];
        double tb = -1.0 * inv * o[a], tt = inv * (dim[a] - o[a]);
        tmin[a] = std::min(tt, tb);
        tmax[a] = std::max(tt, tb);
      }
      double largest_tmin = std::max(std::max(tmin[0], tmin[1]), std::max(tmin[0], tmin[2]));
      double smallest_tmax = std::min(std::min(tmax[0], tmax[1]), std::min(tmax[0], tmax[2]));
      double tnear = std::max(largest_tmin, nearp), tfar = std::min(smallest_tmax, farp);
      double hit[4] = {0, 0, 0, 0};
      if (tnear < tfar) {
        double t = tnear, stepsize = large_step;
        double p[3] = {o[0] + d[0] * t, o[1] + d[1] * t, o[2] + d[2] * t};
        double f_t = rs.interp(p), f_tt = 0;
        if (f_t >= 0) {
          double tb = t;
          long k = 0;
          for (; t < tfar;) {
            double q[3] = {o[0] + d[0] * t, o[1] + d[1] * t, o[2] + d[2] * t};
            f_tt = rs.interp(q);
            if (f_tt < 0) break;
            if (f_tt < 0.8 && stepsize != step) { /* stepsize = step; rebase the march */
              stepsize = step;
              tb = t; k = 0;
            }
            f_t = f_tt;
            ++k;
            t = tb + (double)k * stepsize;
          }
          if (f_tt < 0) {
            t = t + stepsize * f_tt / (f_t - f_tt);
            hit[0] = o[0] + d[0] * t; hit[1] = o[1] + d[1] * t; hit[2] = o[2] + d[2] * t;
            hit[3] = t;
          }
        }
      }
      size_t i = (size_t)y * W + x;
      double* rv = &s->ref_vertex[4 * i];
      double* rn = &s->ref_normal[4 * i];
      if (hit[3] > 0) {
        rv[0] = hit[0]; rv[1] = hit[1]; rv[2] = hit[2]; rv[3] = 1.0;
        double g[3];
        rs.gradient(hit, g);
        double len = std::sqrt(dot3(g, g));
        if (len == 0) {
          rn[0] = rn[1] = rn[2] = rn[3] = 0;
        } else {
          rn[0] = g[0] / len; rn[1] = g[1] / len; rn[2] = g[2] / len; rn[3] = 1.0;
        }
      } else {
        rv[0] = rv[1] = rv[2] = rv[3] = 0;
        rn[0] = rn[1] = rn[2] = rn[3] = 0;
      }
    }
}

/* ---- intensityProjection(): gFusion.cpp:1368-1409 + mip.cs:52-104 -------------------------
 * The raycast's view, slab test and near/far clipping; samples every largeStep = 0.75 mu
 * from tnear while t < tfar (mip.cs:82-100, t = tnear + k * largeStep here); positive
 * samples add to x (the f == 0 branch adds zero to z, the third branch is unreachable);
 * every pixel, misses included, is (sum, 0, 0, 1). */
void intensity_projection(or_session* s, double* rgba) {
  const int W = s->intr.width, H = s->intr.height;
  double invK[16], view[16];
  std::memset(invK, 0, sizeof(invK));
  M(invK, 0, 0) = 1.0 / s->intr.fx; M(invK, 2, 0) = -s->intr.cx / s->intr.fx;
  M(invK, 1, 1) = 1.0 / s->intr.fy; M(invK, 2, 1) = -s->intr.cy / s->intr.fy;
  M(invK, 2, 2) = 1; M(invK, 3, 3) = 1;
  mat4_mul(s->pose, invK, view);
  const double dim[3] = {s->cfg.dim_x, s->cfg.dim_y, s->cfg.dim_z};
  const double large_step = 0.75 * s->cfg.mu;
  const double nearp = s->cfg.near_plane, farp = s->cfg.far_plane;
  RaySampler rs(s);
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      double o[3] = {Mc(view, 3, 0), Mc(view, 3, 1), Mc(view, 3, 2)};
      double pix[3] = {(double)x, (double)y, 1.0};
      double d[3];
      xform(view, pix, 0.0, d);
      double tmin[3], tmax[3];
      for (int a = 0; a < 3; ++a) {
        double inv = 1.0 / d[a];
        double tb = -1.0 * inv * o[a], tt = inv * (dim[a] - o[a]);
        tmin[a] = std::min(tt, tb);
        tmax[a] = std::max(tt, tb);
      }
      double largest_tmin = std::max(std::max(tmin[0], tmin[1]), std::max(tmin[0], tmin[2]));
      double smallest_tmax = std::min(std::min(tmax[0], tmax[1]), std::min(tmax[0], tmax[2]));
      double tnear = std::max(largest_tmin, nearp), tfar = std::min(smallest_tmax, farp);
      double sum = 0.0;
      if (tnear < tfar)
        for (long k = 0;; ++k) {
          const double t = tnear + (double)k * large_step;
          if (!(t < tfar)) break;
          double q[3] = {o[0] + d[0] * t, o[1] + d[1] * t, o[2] + d[2] * t};
          const double f = rs.interp(q);
          if (f > 0) sum += f;
        }
      double* px = &rgba[4 * ((size_t)y * W + x)];
      px[0] = sum; px[1] = 0.0; px[2] = 0.0; px[3] = 1.0;
    }
}

/* ---- marching cubes: histoPyramids.cs classifyCubes/constructHPLevel + traverse ----------- */
const int kHpOff[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 0, 1}, {1, 0, 1},
                          {0, 1, 0}, {1, 1, 0}, {0, 1, 1}, {1, 1, 1}}; /* cubeOffsets */

/* calcNormal (marchingCubes.cs:87-93): cross(v1 - v0, v2 - v0), unnormalised, for the
 * three vertices of a triangle starting at vertex v0i; w = 0. */
void store_face_normal(or_session* s, size_t v0i, const double P[3][3]) {
  double e0[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
  double e1[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
  double n[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0]};
  for (int k = 0; k < 3; ++k) {
    float* o = &s->mc_normals[(v0i + k) * 4];
    o[0] = (float)n[0]; o[1] = (float)n[1]; o[2] = (float)n[2]; o[3] = 0.0f;
  }
}

int mc_histopyramid(or_session* s, double iso) {
  const Volume& V = s->vol;
  const int nx = V.nx, ny = V.ny, nz = V.nz;
  const bool q13 = s->cfg.quirks & KF_Q13_MC_FIRST_SEVEN;
  const bool q15 = s->cfg.quirks & KF_Q15_MC_BORDER_SKIP;
  s->mc_base.assign((size_t)nx * ny * nz, 0u);
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        bool skip;
        if (q15) /* pos <= 10 || pos >= texSize - 10 (histoPyramids.cs:117) */
          skip = x <= 10 || x >= nx - 10 || y <= 10 || y >= ny - 10 || z <= 10 || z >= nz - 10;
        else
          skip = x >= nx - 1 || y >= ny - 1 || z >= nz - 1;
        if (skip) continue;
        double f[8];
        for (int k = 0; k < 8; ++k)
          f[k] = V.raw(V.idx(x + kHpOff[k][0], y + kHpOff[k][1], z + kHpOff[k][2]));
        bool pos = false;
        for (int k = 0; k < (q13 ? 7 : 8); ++k) pos |= f[k] > 0;
        if (!pos) continue; /* written as (0,0) */
        unsigned ci = (unsigned)(f[0] < iso) + (unsigned)(f[1] < iso) * 2 +
                      (unsigned)(f[3] < iso) * 4 + (unsigned)(f[2] < iso) * 8 +
                      (unsigned)(f[4] < iso) * 16 + (unsigned)(f[5] < iso) * 32 +
                      (unsigned)(f[7] < iso) * 64 + (unsigned)(f[6] < iso) * 128;
        s->mc_base[V.idx(x, y, z)] = kf_mc_nr_triangles[ci] | (ci << 16);
      }
  /* pyramid padded to a power of two P (the reference assumes pow2 N, Q16) */
  int P = 1, top = 0;
  while (P < std::max(nx, std::max(ny, nz))) { P <<= 1; ++top; }
  s->mc_levels.assign(top + 1, {});
  for (int k = 1; k <= top; ++k) {
    int D = P >> k;
    std::vector<uint32_t>& Lk = s->mc_levels[k];
    Lk.assign((size_t)D * D * D, 0u);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < D; ++z)
      for (int y = 0; y < D; ++y)
        for (int x = 0; x < D; ++x) {
          uint64_t acc = 0;
          for (int c = 0; c < 8; ++c) {
            int X = 2 * x + kHpOff[c][0], Y = 2 * y + kHpOff[c][1], Z = 2 * z + kHpOff[c][2];
            if (k == 1) {
              if (X < nx && Y < ny && Z < nz) acc += s->mc_base[V.idx(X, Y, Z)] & 0xffff;
            } else {
              int Dp = P >> (k - 1);
              acc += s->mc_levels[k - 1][(size_t)X + (size_t)Dp * ((size_t)Y + (size_t)Dp * Z)];
            }
          }
          Lk[(size_t)x + (size_t)D * ((size_t)y + (size_t)D * z)] = (uint32_t)acc;
        }
  }
  uint32_t total = top > 0 ? s->mc_levels[top][0] : (s->mc_base[0] & 0xffff);
  s->mc_triangles = total;
  s->mc_vertices.assign((size_t)total * 3 * 4, 0.0f);
  s->mc_normals.assign((size_t)total * 3 * 4, 0.0f);
  auto level_val = [&](int k, int x, int y, int z) -> uint32_t {
    if (k == 0) {
      if (x >= nx || y >= ny || z >= nz) return 0;
      return s->mc_base[V.idx(x, y, z)] & 0xffff;
    }
    int D = P >> k;
    if (x >= D || y >= D || z >= D) return 0;
    return s->mc_levels[k][(size_t)x + (size_t)D * ((size_t)y + (size_t)D * z)];
  };
  /* traverseHPLevel (traverseHistoPyramids.cs:136-260), one triangle per iteration */
#pragma omp parallel for schedule(static)
  for (long t = 0; t < (long)total; ++t) {
    uint32_t target = (uint32_t)t;
    int cx = 0, cy = 0, cz = 0;
    uint32_t w = 0;
    for (int k = top - 1; k >= 0; --k) { /* scanHPLevel, :54-119 */
      uint32_t nb[8];
      for (int c = 0; c < 8; ++c)
        nb[c] = level_val(k, cx + kHpOff[c][0], cy + kHpOff[c][1], cz + kHpOff[c][2]);
      uint32_t acc = w;
      int sel = 0;
      uint32_t add = 0;
      for (int c = 0; c < 7; ++c) {
        acc += nb[c];
        if (acc <= target) { ++sel; add += nb[c]; }
      }
      cx = (cx + kHpOff[sel][0]) * 2;
      cy = (cy + kHpOff[sel][1]) * 2;
      cz = (cz + kHpOff[sel][2]) * 2;
      w += add;
    }
    cx /= 2; cy /= 2; cz /= 2;
    unsigned ci = s->mc_base[V.idx(cx, cy, cz)] >> 16;
    int j = (int)(target - w);
    double P[3][3];
    for (int k = 0; k < 3; ++k) {
      int edge = kf_mc_tri_table[ci * 16 + 3 * j + k];
      const uint8_t* o = &kf_mc_offsets3[edge * 6];
      int p0[3] = {cx + o[0], cy + o[1], cz + o[2]};
      int p1[3] = {cx + o[3], cy + o[4], cz + o[5]};
      double v0 = V.raw(V.idx(p0[0], p0[1], p0[2]));
      double v1 = V.raw(V.idx(p1[0], p1[1], p1[2]));
      double a = (iso - v0) / (v1 - v0);
      if (a > 1 || a < 0) a = 0.5;
      float* out = &s->mc_vertices[((size_t)t * 3 + k) * 4];
      for (int q = 0; q < 3; ++q) {
        P[k][q] = p0[q] * (1.0 - a) + p1[q] * a;
        out[q] = (float)P[k][q];
      }
      out[3] = 0.0f;
    }
    store_face_normal(s, (size_t)t * 3, P);
  }
  return KF_OK;
}

/* ---- classic path: marchingCubes.cs:102-305 with a full-size exclusive scan ------------- */
const int kBourke[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                           {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
const int kBourkeEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

int mc_scan(or_session* s, double iso) {
  const Volume& V = s->vol;
  const int nx = V.nx, ny = V.ny, nz = V.nz;
  const bool q13 = s->cfg.quirks & KF_Q13_MC_FIRST_SEVEN;
  size_t n = V.count();
  std::vector<uint32_t> verts(n, 0u), cis(n, 0u);
  auto sample = [&](int x, int y, int z) { /* sampleVolume clamps to gridSize-1, :70-78 */
    x = std::min(x, nx - 1); y = std::min(y, ny - 1); z = std::min(z, nz - 1);
    return V.raw(V.idx(x, y, z));
  };
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        double f[8];
        for (int k = 0; k < 8; ++k) f[k] = sample(x + kBourke[k][0], y + kBourke[k][1], z + kBourke[k][2]);
        bool pos = false;
        for (int k = 0; k < (q13 ? 7 : 8); ++k) pos |= f[k] > 0;
        size_t i = V.idx(x, y, z);
        if (!pos) continue;
        unsigned ci = 0;
        for (int k = 0; k < 8; ++k) ci |= (unsigned)(f[k] < iso) << k;
        verts[i] = kf_mc_num_verts[ci];
        cis[i] = ci;
      }
  std::vector<uint32_t> scan(n);
  uint32_t total_verts = 0;
  or_prefix_sum_u32(verts.data(), scan.data(), n, &total_verts);
  s->mc_base.assign(n, 0u);
  for (size_t i = 0; i < n; ++i) s->mc_base[i] = (verts[i] / 3) | (cis[i] << 16);
  s->mc_levels.clear();
  s->mc_triangles = total_verts / 3;
  s->mc_vertices.assign((size_t)total_verts * 4, 0.0f);
  s->mc_normals.assign((size_t)total_verts * 4, 0.0f);
  /* Q24: the shader's units, corners at -1 + gridPos * voxelSize (launchGenerateTriangles,
   * marchingCubes.cs:205-220), voxelSize = mCubeConfig's 1000 * dim / size */
  const bool q24 = s->cfg.quirks & KF_Q24_MC_SHADER_UNITS;
  const double vs[3] = {1000.0 * s->cfg.dim_x / nx, 1000.0 * s->cfg.dim_y / ny, 1000.0 * s->cfg.dim_z / nz};
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        size_t i = V.idx(x, y, z);
        if (!verts[i]) continue;
        double f[8];
        for (int k = 0; k < 8; ++k) f[k] = sample(x + kBourke[k][0], y + kBourke[k][1], z + kBourke[k][2]);
        unsigned ci = cis[i];
        const int g[3] = {x, y, z};
        for (unsigned v = 0; v < verts[i]; v += 3) {
          double P[3][3];
          for (int k = 0; k < 3; ++k) {
            int e = kf_mc_tri_table[ci * 16 + v + k];
            int a = kBourkeEdge[e][0], b = kBourkeEdge[e][1];
            double t = (iso - f[a]) / (f[b] - f[a]); /* vertexInterp, :81-85 */
            for (int q = 0; q < 3; ++q) {
              double pa = g[q] + kBourke[a][q], pb = g[q] + kBourke[b][q];
              if (q24) {
                pa = -1.0 + g[q] * vs[q] + kBourke[a][q] * vs[q];
                pb = -1.0 + g[q] * vs[q] + kBourke[b][q] * vs[q];
              }
              P[k][q] = pa * (1.0 - t) + pb * t;
            }
          }
          store_face_normal(s, (size_t)scan[i] + v, P);
          for (int k = 0; k < 3; ++k) {
            float* out = &s->mc_vertices[((size_t)scan[i] + v + k) * 4];
            if (q24) { /* pos[index] of :290-299: / 128 * voxelSize.x, z negated */
              out[0] = (float)(P[k][0] / 128.0 * vs[0]);
              out[1] = (float)(P[k][1] / 128.0 * vs[0]);
              out[2] = (float)(-(P[k][2] / 128.0) * vs[0]);
            } else {
              out[0] = (float)P[k][0]; out[1] = (float)P[k][1]; out[2] = (float)P[k][2];
            }
            out[3] = 1.0f;
          }
        }
      }
  return KF_OK;
}

/* ---- welded mesh: the export form of the CUDA path, restated --------------------------
 * Interior cubes [0, n-2]^3 in the classic path's Bourke order and case table; a triangle
 * vertex on cube edge e belongs to the edge's lower voxel and axis; used edges are numbered
 * in voxel order, then axis; position = voxel-index point + 0.5, times dim / size (metres);
 * normal = the unit interpolation of the central-difference gradients at the two voxels. */
int mc_mesh(or_session* s, double iso) {
  const Volume& V = s->vol;
  const int nx = V.nx, ny = V.ny, nz = V.nz;
  const bool q13 = s->cfg.quirks & KF_Q13_MC_FIRST_SEVEN;
  const size_t n = V.count();
  static const int owner[12][4] = {{0, 0, 0, 0}, {1, 0, 0, 1}, {0, 1, 0, 0}, {0, 0, 0, 1},
                                   {0, 0, 1, 0}, {1, 0, 1, 1}, {0, 1, 1, 0}, {0, 0, 1, 1},
                                   {0, 0, 0, 2}, {1, 0, 0, 2}, {1, 1, 0, 2}, {0, 1, 0, 2}};
  std::vector<uint8_t> mark(n, 0);
  std::vector<std::pair<size_t, unsigned>> cubes; /* (voxel, case) of cubes with triangles */
  for (int z = 0; z + 1 < nz; ++z)
    for (int y = 0; y + 1 < ny; ++y)
      for (int x = 0; x + 1 < nx; ++x) {
        double f[8];
        for (int k = 0; k < 8; ++k) f[k] = V.raw(V.idx(x + kBourke[k][0], y + kBourke[k][1], z + kBourke[k][2]));
        bool pos = false;
        for (int k = 0; k < (q13 ? 7 : 8); ++k) pos |= f[k] > 0;
        if (!pos) continue;
        unsigned ci = 0;
        for (int k = 0; k < 8; ++k) ci |= (unsigned)(f[k] < iso) << k;
        if (!kf_mc_num_verts[ci]) continue;
        cubes.emplace_back(V.idx(x, y, z), ci);
        for (int k = 0; k < kf_mc_num_verts[ci]; ++k) {
          const int* o = owner[kf_mc_tri_table[ci * 16 + k]];
          mark[V.idx(x + o[0], y + o[1], z + o[2])] |= (uint8_t)(1u << o[3]);
        }
      }
  std::vector<uint32_t> id(3 * n, 0xffffffffu);
  uint32_t nv = 0;
  for (size_t v = 0; v < n; ++v)
    for (int a = 0; a < 3; ++a)
      if (mark[v] >> a & 1) id[3 * v + a] = nv++;
  s->mesh_pos.assign((size_t)nv * 3, 0.0f);
  s->mesh_nrm.assign((size_t)nv * 3, 0.0f);
  const int dims[3] = {nx, ny, nz};
  const double dimm[3] = {s->cfg.dim_x, s->cfg.dim_y, s->cfg.dim_z};
  auto val = [&](int x, int y, int z) {
    x = std::min(std::max(x, 0), nx - 1);
    y = std::min(std::max(y, 0), ny - 1);
    z = std::min(std::max(z, 0), nz - 1);
    return V.raw(V.idx(x, y, z));
  };
  auto grad = [&](int x, int y, int z, double* g) {
    g[0] = (val(x + 1, y, z) - val(x - 1, y, z)) * 0.5 * nx / dimm[0];
    g[1] = (val(x, y + 1, z) - val(x, y - 1, z)) * 0.5 * ny / dimm[1];
    g[2] = (val(x, y, z + 1) - val(x, y, z - 1)) * 0.5 * nz / dimm[2];
  };
  for (size_t v = 0; v < n; ++v)
    for (int a = 0; a < 3; ++a) {
      if (!(mark[v] >> a & 1)) continue;
      const uint32_t i = id[3 * v + a];
      int p0[3] = {(int)(v % nx), (int)((v / nx) % ny), (int)(v / ((size_t)nx * ny))};
      int p1[3] = {p0[0], p0[1], p0[2]};
      p1[a] += 1;
      const double f0 = V.raw(V.idx(p0[0], p0[1], p0[2])), f1 = V.raw(V.idx(p1[0], p1[1], p1[2]));
      const double t = (iso - f0) / (f1 - f0);
      double g0[3], g1[3], g[3];
      grad(p0[0], p0[1], p0[2], g0);
      grad(p1[0], p1[1], p1[2], g1);
      for (int k = 0; k < 3; ++k) {
        const double p = p0[k] + t * (p1[k] - p0[k]);
        s->mesh_pos[3 * i + k] = (float)((p + 0.5) * dimm[k] / dims[k]);
        g[k] = g0[k] + t * (g1[k] - g0[k]);
      }
      const double len = std::sqrt(dot3(g, g));
      for (int k = 0; k < 3; ++k) s->mesh_nrm[3 * i + k] = (float)(len > 0 ? g[k] / len : 0.0);
    }
  /* each triangle (a, b, c) of the table is stored as (a, c, b): counter-clockwise seen
   * from the positive side, its facet normal along the gradient */
  s->mesh_idx.clear();
  for (const auto& c : cubes) {
    const size_t v = c.first;
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((size_t)nx * ny));
    for (int k = 0; k < kf_mc_num_verts[c.second]; k += 3) {
      uint32_t t[3];
      for (int q = 0; q < 3; ++q) {
        const int* o = owner[kf_mc_tri_table[c.second * 16 + k + q]];
        t[q] = id[3 * V.idx(x + o[0], y + o[1], z + o[2]) + o[3]];
      }
      s->mesh_idx.push_back(t[0]);
      s->mesh_idx.push_back(t[2]);
      s->mesh_idx.push_back(t[1]);
    }
  }
  s->mesh_valid = 1;
  return KF_OK;
}

}  // namespace

/* ====================================================================================== */
extern "C" {

int or_create(const kf_config* cfg, const kf_intrinsics* intr, or_session** out) {
  if (!cfg || !intr || !out) return KF_ERR_INVALID_ARGUMENT;
  if (cfg->nx < 4 || cfg->ny < 4 || cfg->nz < 4 || intr->width < 8 || intr->height < 8)
    return KF_ERR_INVALID_ARGUMENT;
  or_session* s = new or_session();
  s->cfg = *cfg;
  s->intr = *intr;
  s->vol.alloc(cfg->storage, cfg->nx, cfg->ny, cfg->nz);
  level_setup(s);
  double I[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  std::memcpy(s->pose, I, sizeof(I));
  std::memcpy(s->pose_eig, I, sizeof(I));
  std::memcpy(s->raycast_pose, I, sizeof(I));
  std::memset(s->last_sums, 0, sizeof(s->last_sums));
  *out = s;
  return KF_OK;
}

int or_destroy(or_session* s) { delete s; return KF_OK; }

int or_reset_pose(or_session* s, const double pose[16]) {
  /* resetPose (gFusion.cpp:275-287): with Q19 m_pose_eig = identity + translation only */
  std::memcpy(s->pose, pose, 16 * sizeof(double));
  if (s->cfg.quirks & KF_Q19_EIG_TRANSLATION) {
    double I[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    std::memcpy(s->pose_eig, I, sizeof(I));
    s->pose_eig[12] = pose[12]; s->pose_eig[13] = pose[13]; s->pose_eig[14] = pose[14];
  } else {
    std::memcpy(s->pose_eig, pose, 16 * sizeof(double));
  }
  for (int i = 0; i < 6; ++i) s->cum_twist[i] = 0;
  return KF_OK;
}

int or_reset(or_session* s, const double pose[16], int delete_flag) {
  (void)delete_flag;
  s->vol.zero();
  s->library.clear();
  or_reset_pose(s, pose);
  /* the app's "Reset Volume" button (kinect.cpp:446-477): reset = true, counter = 0,
   * raycast() of the empty volume (all zeros) */
  s->reset_window = true;
  s->counter = 0;
  std::memcpy(s->raycast_pose, pose, 16 * sizeof(double));
  std::fill(s->ref_vertex.begin(), s->ref_vertex.end(), 0.0);
  std::fill(s->ref_normal.begin(), s->ref_normal.end(), 0.0);
  return KF_OK;
}

int or_set_pose(or_session* s, const double pose[16]) { std::memcpy(s->pose, pose, 128); return KF_OK; }
int or_get_pose(or_session* s, double pose[16]) { std::memcpy(pose, s->pose, 128); return KF_OK; }
int or_get_pose_eig(or_session* s, double pose[16]) { std::memcpy(pose, s->pose_eig, 128); return KF_OK; }
int or_set_pose_eig(or_session* s, const double pose[16]) { std::memcpy(s->pose_eig, pose, 128); return KF_OK; }

int or_depth_to_vertex_f32(or_session* s, const float* depth_mm) {
  prepare_depth(s, depth_mm);
  depth_to_vertex(s);
  return KF_OK;
}

int or_depth_to_vertex_u16(or_session* s, const uint16_t* depth_mm) {
  std::vector<float> f(s->lv[0].depth.size());
  for (size_t i = 0; i < f.size(); ++i) f[i] = depth_mm[i];
  prepare_depth(s, f.data());
  depth_to_vertex(s);
  return KF_OK;
}

int or_set_depth_undistortion(or_session* s, const float ir[9]) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  if (!ir) {
    s->undistort = false;
    return KF_OK;
  }
  const int W = s->lv[0].w, H = s->lv[0].h;
  s->undistort_map.assign((size_t)W * H, -1);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) s->undistort_map[(size_t)y * W + x] = undistort_index(ir, x, y, W, H);
  s->undistort = true;
  return KF_OK;
}

int or_set_depth_filter(or_session* s, int enable) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  s->depth_filter = enable != 0;
  return KF_OK;
}

int or_get_undistortion_map(or_session* s, int32_t* map) {
  if (!s || !map || !s->undistort) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(map, s->undistort_map.data(), s->undistort_map.size() * sizeof(int32_t));
  return KF_OK;
}

int or_vertex_to_normal(or_session* s) { vertex_to_normal(s); return KF_OK; }

int or_track_icp(or_session* s, int* tracked) {
  bool t = track_icp(s);
  if (tracked) *tracked = t;
  return KF_OK;
}

int or_track_sdf(or_session* s, int* tracked) {
  bool t = track_sdf(s);
  if (tracked) *tracked = t;
  return KF_OK;
}

int or_recover_pose(or_session* s, int* found) {
  bool f = recover_pose(s);
  if (found) *found = f;
  return KF_OK;
}

int or_get_alignment_energy(or_session* s, double* ae) { *ae = s->ae; return KF_OK; }
int or_get_reduction(or_session* s, double sums[32]) { std::memcpy(sums, s->last_sums, 256); return KF_OK; }

int or_icp_reduce_once(or_session* s, int level, double sums[32]) {
  if (level < 0 || level > 2) return KF_ERR_INVALID_ARGUMENT;
  icp_track_reduce(s, level, sums);
  return KF_OK;
}

int or_sdf_reduce_once(or_session* s, int level, const double T[16], double sums[32]) {
  if (level < 0 || level > 2) return KF_ERR_INVALID_ARGUMENT;
  sdf_track_reduce(s, level, T, sums);
  return KF_OK;
}

int or_integrate(or_session* s) { integrate(s); return KF_OK; }
int or_raycast(or_session* s) { raycast(s); return KF_OK; }

int or_intensity_projection(or_session* s, double* rgba) {
  if (!s || !rgba) return KF_ERR_INVALID_ARGUMENT;
  intensity_projection(s, rgba);
  return KF_OK;
}

int or_frame_step_u16(or_session* s, const uint16_t* depth_mm, int* tracked_out) {
  /* kinect.cpp:654-695 with trackDepthToPoint / trackDepthToVolume from cfg.tracking */
  or_depth_to_vertex_u16(s, depth_mm);
  vertex_to_normal(s);
  bool tracked = (s->cfg.tracking == KF_TRACK_SDF) ? track_sdf(s) : track_icp(s);
  int every = s->cfg.integrate_every > 0 ? s->cfg.integrate_every : 1;
  if ((tracked && (s->counter % every) == 0) || s->reset_window) {
    integrate(s);
    if (s->counter > 2) s->reset_window = false;
  }
  if (!tracked) recover_pose(s);
  s->counter++;
  raycast(s);
  if (tracked_out) *tracked_out = tracked;
  return KF_OK;
}

int or_get_raycast(or_session* s, double* v, double* n) {
  if (v) std::memcpy(v, s->ref_vertex.data(), s->ref_vertex.size() * 8);
  if (n) std::memcpy(n, s->ref_normal.data(), s->ref_normal.size() * 8);
  return KF_OK;
}

int or_set_raycast(or_session* s, const double* v, const double* n) {
  std::memcpy(s->ref_vertex.data(), v, s->ref_vertex.size() * 8);
  std::memcpy(s->ref_normal.data(), n, s->ref_normal.size() * 8);
  return KF_OK;
}

int or_get_vertex_map(or_session* s, int l, double* v) {
  if (l < 0 || l > 2) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(v, s->lv[l].vertex.data(), s->lv[l].vertex.size() * 8);
  return KF_OK;
}

int or_get_normal_map(or_session* s, int l, double* n) {
  if (l < 0 || l > 2) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(n, s->lv[l].normal.data(), s->lv[l].normal.size() * 8);
  return KF_OK;
}

int or_set_vertex_normal_map(or_session* s, int l, const double* v, const double* n) {
  if (l < 0 || l > 2) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(s->lv[l].vertex.data(), v, s->lv[l].vertex.size() * 8);
  std::memcpy(s->lv[l].normal.data(), n, s->lv[l].normal.size() * 8);
  return KF_OK;
}

int or_get_depth_map(or_session* s, int l, double* d) {
  if (l < 0 || l > 2) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(d, s->lv[l].depth.data(), s->lv[l].depth.size() * 8);
  return KF_OK;
}

int or_get_track_status(or_session* s, int l, int32_t* st) {
  if (l < 0 || l > 2) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(st, s->lv[l].status.data(), s->lv[l].status.size() * 4);
  return KF_OK;
}

int or_copy_volume_to_host(or_session* s, void* dst, uint64_t bytes) {
  if (bytes != s->vol.bytes()) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(dst, s->vol.buf.data(), bytes);
  return KF_OK;
}

int or_copy_volume_from_host(or_session* s, const void* src, uint64_t bytes) {
  if (bytes != s->vol.bytes()) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(s->vol.buf.data(), src, bytes);
  return KF_OK;
}

int or_get_pose_library_size(or_session* s, int* n) { *n = (int)s->library.size(); return KF_OK; }
int or_get_cum_twist(or_session* s, double t[6]) { std::memcpy(t, s->cum_twist, 48); return KF_OK; }

int or_mc_extract(or_session* s, float iso, int method, uint32_t* n_tri) {
  int rc = (method == KF_MC_SCAN) ? mc_scan(s, iso) : mc_histopyramid(s, iso);
  s->mc_valid = (rc == KF_OK);
  if (n_tri) *n_tri = s->mc_triangles;
  return rc;
}

int or_mc_copy_vertices(or_session* s, float* v, uint64_t max_vertices) {
  uint64_t n = (uint64_t)s->mc_triangles * 3;
  if (max_vertices < n) return KF_ERR_CAPACITY;
  std::memcpy(v, s->mc_vertices.data(), n * 16);
  return KF_OK;
}

int or_mc_extract_mesh(or_session* s, float iso, uint32_t* nv, uint32_t* nt) {
  int rc = mc_mesh(s, iso);
  *nv = (uint32_t)(s->mesh_pos.size() / 3);
  *nt = (uint32_t)(s->mesh_idx.size() / 3);
  return rc;
}

int or_mc_copy_mesh(or_session* s, float* pos, float* nrm, uint32_t* idx) {
  if (!s->mesh_valid) return KF_ERR_STATE;
  std::memcpy(pos, s->mesh_pos.data(), s->mesh_pos.size() * 4);
  std::memcpy(nrm, s->mesh_nrm.data(), s->mesh_nrm.size() * 4);
  std::memcpy(idx, s->mesh_idx.data(), s->mesh_idx.size() * 4);
  return KF_OK;
}

int or_mc_copy_normals(or_session* s, float* n, uint64_t max_vertices) {
  uint64_t cnt = (uint64_t)s->mc_triangles * 3;
  if (max_vertices < cnt) return KF_ERR_CAPACITY;
  std::memcpy(n, s->mc_normals.data(), cnt * 16);
  return KF_OK;
}

int or_mc_copy_base_level(or_session* s, uint32_t* base, uint64_t count) {
  if (count != s->mc_base.size()) return KF_ERR_INVALID_ARGUMENT;
  std::memcpy(base, s->mc_base.data(), count * 4);
  return KF_OK;
}

int or_mc_export_stl(or_session* s, const char* path) {
  /* exportMesh (mcubes.cpp:429-509): 80-byte header, uint32 count, then per triangle the
   * normal (1,1,1), three vertices and a zero uint16 attribute. */
  if (!s->mc_valid) return KF_ERR_STATE;
  std::ofstream f(path, std::ios::binary);
  if (!f) return KF_ERR_IO;
  char hdr[80];
  std::memset(hdr, 0, sizeof(hdr));
  f.write(hdr, 80);
  uint32_t T = s->mc_triangles;
  uint32_t count = (s->cfg.quirks & KF_Q18_STL_COUNT_X4) ? 4 * T : T;
  f.write((const char*)&count, 4);
  const float nrm[3] = {1.0f, 1.0f, 1.0f};
  const uint16_t attr = 0;
  for (uint32_t t = 0; t < T; ++t) {
    f.write((const char*)nrm, 12);
    for (int k = 0; k < 3; ++k) f.write((const char*)&s->mc_vertices[((size_t)t * 3 + k) * 4], 12);
    f.write((const char*)&attr, 2);
  }
  return f.good() ? KF_OK : KF_ERR_IO;
}

int or_mc_export_ply(or_session* s, const char* path) {
  /* exportPointCloud (mcubes.cpp:391-427): ASCII PLY of the vertex buffer */
  if (!s->mc_valid) return KF_ERR_STATE;
  FILE* f = std::fopen(path, "w");
  if (!f) return KF_ERR_IO;
  uint64_t n = (uint64_t)s->mc_triangles * 3;
  std::fprintf(f, "ply\nformat ascii 1.0\nelement vertex %llu\nproperty float x\n"
               "property float y\nproperty float z\nend_header\n", (unsigned long long)n);
  for (uint64_t i = 0; i < n; ++i)
    std::fprintf(f, "%g %g %g\n", s->mc_vertices[i * 4], s->mc_vertices[i * 4 + 1],
                 s->mc_vertices[i * 4 + 2]);
  int bad = std::ferror(f);
  std::fclose(f);
  return bad ? KF_ERR_IO : KF_OK;
}

}  // extern "C"
