// mhc_device.cuh -- device-side arithmetic shared by every MaHyCo kernel.
//
// All kernels are compiled with --fmad=false: every expression below rounds
// exactly like the reference's x86-64 build (no contraction), so results can
// be compared with the CPU oracle operation by operation.  Vector operations
// follow Arcane's Real3 helpers (component-wise, left-to-right sums).
#pragma once
#include <cstdint>
#include <cmath>

namespace mhc {

struct R3 {
  double x, y, z;
};
__device__ __forceinline__ R3 operator+(R3 a, R3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ R3 operator-(R3 a, R3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ R3 operator*(double s, R3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ R3 operator*(R3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ R3 operator/(R3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ R3 operator-(R3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ double dot(R3 a, R3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// math::vecMul
__device__ __forceinline__ R3 vecmul(R3 u, R3 v) {
  return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
__device__ __forceinline__ double norm(R3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ double comp(R3 a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }
// MahycoModule::produit
__device__ __forceinline__ double produit(double A, double B, double C, double D) { return A * B - C * D; }
// Arcane math::min / math::max
__device__ __forceinline__ double amin(double a, double b) { return (a < b) ? a : b; }
__device__ __forceinline__ double amax(double a, double b) { return (a < b) ? b : a; }
// std::min / std::max
__host__ __device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// ---------------------------------------------------------------------------
// correctly rounded powers
// ---------------------------------------------------------------------------
// Error-free product a*b = p + e (Dekker/Ogita-Rump-Oishi TwoProduct, using
// the fused multiply-add as the exact remainder).
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = fma(a, b, -p);
}

// x^3 rounded once: the exact cube is the sum of four doubles.
__device__ __forceinline__ double cube_rn(double x) {
  double s, sl, t, tl, u, ul;
  two_prod(x, x, s, sl);
  two_prod(s, x, t, tl);
  two_prod(sl, x, u, ul);
  return t + (tl + (u + ul));
}

// x^y for y = the double nearest to 1/3 (the reference writes pow(V, 1./3.)).
// With y = 1/3 - d, d = 2^-54/3 exactly, x^y = cbrt(x) * exp(-d ln x).
// cbrt(x) is refined to double-double by one Newton step on r^3 = x with an
// exact residual, the tiny factor exp(-d ln x) ~ 1 - d ln x is applied to
// first order (the second-order term is below 2^-100), and the double-double
// is rounded once.  The result is the correctly rounded x^y except when x^y
// lies within ~2^-90 relative of a rounding boundary.
__device__ __forceinline__ double pow_one_third(double x) {
  if (!(x > 0.0) || isinf(x)) return pow(x, 1. / 3.);
  double r = cbrt(x);
  double s, sl, t, tl;
  two_prod(r, r, s, sl);
  two_prod(s, r, t, tl);
  double res = ((x - t) - tl) - sl * r;   // x - r^3, exact to ~2^-106 relative
  double c_lo = res / (3.0 * s);         // cbrt(x) = r + c_lo
  const double d = (1.0 / 3.0) * 0x1p-54; // 1/3 - double(1/3)
  double corr = c_lo - r * (d * log(x));
  return r + corr;
}

// x^y for y = the double nearest to 5/3 (NewHypoModelService.cc:123 writes
// pow(J, 5./3.)).  y = 5/3 + d, d = 2^-52/3 exactly, so x^y = x c^2 x^d with
// c = cbrt(x) refined to double-double as above; x c^2 is formed as a
// double-double (TwoProduct), the factor x^d ~ 1 + d ln x applied to first
// order, and the sum rounded once: the correctly rounded x^y except within
// ~2^-90 relative of a rounding boundary.
__device__ __forceinline__ double pow_five_thirds(double x) {
  if (!(x > 0.0) || isinf(x)) return pow(x, 5. / 3.);
  double r = cbrt(x);
  double s, sl, t, tl;
  two_prod(r, r, s, sl);
  two_prod(s, r, t, tl);
  const double c_lo = (((x - t) - tl) - sl * r) / (3.0 * s);  // cbrt(x) = r + c_lo
  double q, ql;
  two_prod(x, s, q, ql);                                        // x r^2 = q + ql
  const double d = (1.0 / 3.0) * 0x1p-52;                       // double(5/3) - 5/3
  const double corr = (ql + x * (sl + 2.0 * r * c_lo)) + q * (d * log(x));
  return q + corr;
}

// ---------------------------------------------------------------------------
// structured mesh indexing (Arcane cartesian generator numbering)
// ---------------------------------------------------------------------------
struct Mesh {
  int dim;
  int ncx, ncy, ncz;   // cells per direction (ncz = 1 in 2D)
  int nnx, nny, nnz;   // nodes per direction (nnz = 1 in 2D)
  long long ncell, nnode;
  double o[3];         // origin
  double h[3];         // L/n per direction
};

// linear ids in 32-bit arithmetic: a case has fewer than 2^31 nodes
// (checked at creation), and every offset into a field array stays 64-bit
__device__ __forceinline__ long long cell_id(const Mesh& M, int i, int j, int k) {
  return (long long)(unsigned)(i + M.ncx * (j + M.ncy * k));
}
__device__ __forceinline__ long long node_id(const Mesh& M, int i, int j, int k) {
  return (long long)(unsigned)(i + M.nnx * (j + M.nny * k));
}
// (i, j, k) of a linear id, in unsigned 32-bit arithmetic (ids < 2^31):
// a 64-bit division is a long emulated sequence, a 32-bit one a few
// instructions
__device__ __forceinline__ void cell_ijk(const Mesh& M, long long c, int& i, int& j, int& k) {
  const unsigned u = (unsigned)c, nx = (unsigned)M.ncx, ny = (unsigned)M.ncy;
  const unsigned r = u / nx;
  i = (int)(u - r * nx);
  k = (int)(r / ny);
  j = (int)(r - (unsigned)k * ny);
}
__device__ __forceinline__ void node_ijk(const Mesh& M, long long n, int& i, int& j, int& k) {
  const unsigned u = (unsigned)n, nx = (unsigned)M.nnx, ny = (unsigned)M.nny;
  const unsigned r = u / nx;
  i = (int)(u - r * nx);
  k = (int)(r / ny);
  j = (int)(r - (unsigned)k * ny);
}
// initial (Euler) node position: origin + i*(L/n)
__device__ __forceinline__ R3 node_x0(const Mesh& M, int i, int j, int k) {
  return {M.o[0] + i * M.h[0], M.o[1] + j * M.h[1], M.dim == 3 ? M.o[2] + k * M.h[2] : 0.};
}

// Hexa8 / Quad4 local node offsets
__device__ __forceinline__ void local_node_offset(int l, int& di, int& dj, int& dk) {
  di = (l == 1 || l == 2 || l == 5 || l == 6) ? 1 : 0;
  dj = (l == 2 || l == 3 || l == 6 || l == 7) ? 1 : 0;
  dk = (l >= 4) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// corner normals
// ---------------------------------------------------------------------------
// face centres of a hexahedron (MahycoModule.cc:1117-1122)
__device__ __forceinline__ void hex_face_centres(const R3* coord, R3* fc) {
  fc[0] = 0.25 * (coord[0] + coord[3] + coord[2] + coord[1]);
  fc[1] = 0.25 * (coord[0] + coord[4] + coord[7] + coord[3]);
  fc[2] = 0.25 * (coord[0] + coord[1] + coord[5] + coord[4]);
  fc[3] = 0.25 * (coord[4] + coord[5] + coord[6] + coord[7]);
  fc[4] = 0.25 * (coord[1] + coord[2] + coord[6] + coord[5]);
  fc[5] = 0.25 * (coord[2] + coord[3] + coord[7] + coord[6]);
}

// MahycoModule::computeCQs (MahycoModule.cc:1869-1932)
__device__ __forceinline__ void cqs3(const R3* nc, const R3* fc, R3* out) {
  const R3 c0 = fc[0], c1 = fc[1], c2 = fc[2], c3 = fc[3], c4 = fc[4], c5 = fc[5];
  const R3 n1a04 = 0.5 * vecmul(nc[0] - c0, nc[3] - c0);
  const R3 n1a03 = 0.5 * vecmul(nc[3] - c0, nc[2] - c0);
  const R3 n1a02 = 0.5 * vecmul(nc[2] - c0, nc[1] - c0);
  const R3 n1a01 = 0.5 * vecmul(nc[1] - c0, nc[0] - c0);
  const R3 n2a05 = 0.5 * vecmul(nc[0] - c1, nc[4] - c1);
  const R3 n2a12 = 0.5 * vecmul(nc[4] - c1, nc[7] - c1);
  const R3 n2a08 = 0.5 * vecmul(nc[7] - c1, nc[3] - c1);
  const R3 n2a04 = 0.5 * vecmul(nc[3] - c1, nc[0] - c1);
  const R3 n3a01 = 0.5 * vecmul(nc[0] - c2, nc[1] - c2);
  const R3 n3a06 = 0.5 * vecmul(nc[1] - c2, nc[5] - c2);
  const R3 n3a09 = 0.5 * vecmul(nc[5] - c2, nc[4] - c2);
  const R3 n3a05 = 0.5 * vecmul(nc[4] - c2, nc[0] - c2);
  const R3 n4a09 = 0.5 * vecmul(nc[4] - c3, nc[5] - c3);
  const R3 n4a10 = 0.5 * vecmul(nc[5] - c3, nc[6] - c3);
  const R3 n4a11 = 0.5 * vecmul(nc[6] - c3, nc[7] - c3);
  const R3 n4a12 = 0.5 * vecmul(nc[7] - c3, nc[4] - c3);
  const R3 n5a02 = 0.5 * vecmul(nc[1] - c4, nc[2] - c4);
  const R3 n5a07 = 0.5 * vecmul(nc[2] - c4, nc[6] - c4);
  const R3 n5a10 = 0.5 * vecmul(nc[6] - c4, nc[5] - c4);
  const R3 n5a06 = 0.5 * vecmul(nc[5] - c4, nc[1] - c4);
  const R3 n6a03 = 0.5 * vecmul(nc[2] - c5, nc[3] - c5);
  const R3 n6a08 = 0.5 * vecmul(nc[3] - c5, nc[7] - c5);
  const R3 n6a11 = 0.5 * vecmul(nc[7] - c5, nc[6] - c5);
  const R3 n6a07 = 0.5 * vecmul(nc[6] - c5, nc[2] - c5);
  const double t = 1. / 12.;
  out[0] = (5. * (n1a01 + n1a04 + n2a04 + n2a05 + n3a05 + n3a01) + (n1a02 + n1a03 + n2a08 + n2a12 + n3a06 + n3a09)) * t;
  out[1] = (5. * (n1a01 + n1a02 + n3a01 + n3a06 + n5a06 + n5a02) + (n1a04 + n1a03 + n3a09 + n3a05 + n5a10 + n5a07)) * t;
  out[2] = (5. * (n1a02 + n1a03 + n5a07 + n5a02 + n6a07 + n6a03) + (n1a01 + n1a04 + n5a06 + n5a10 + n6a11 + n6a08)) * t;
  out[3] = (5. * (n1a03 + n1a04 + n2a08 + n2a04 + n6a08 + n6a03) + (n1a01 + n1a02 + n2a05 + n2a12 + n6a07 + n6a11)) * t;
  out[4] = (5. * (n2a05 + n2a12 + n3a05 + n3a09 + n4a09 + n4a12) + (n2a08 + n2a04 + n3a01 + n3a06 + n4a10 + n4a11)) * t;
  out[5] = (5. * (n3a06 + n3a09 + n4a09 + n4a10 + n5a10 + n5a06) + (n3a01 + n3a05 + n4a12 + n4a11 + n5a07 + n5a02)) * t;
  out[6] = (5. * (n4a11 + n4a10 + n5a10 + n5a07 + n6a07 + n6a11) + (n4a12 + n4a09 + n5a06 + n5a02 + n6a03 + n6a08)) * t;
  out[7] = (5. * (n2a08 + n2a12 + n4a12 + n4a11 + n6a11 + n6a08) + (n2a04 + n2a05 + n4a09 + n4a10 + n6a07 + n6a03)) * t;
}

// 2D corner normals (MahycoModule.cc:1128-1146)
__device__ __forceinline__ void cqs2(const R3* c4, R3* out) {
  R3 coord[5] = {c4[0], c4[1], c4[2], c4[3], c4[0]};
  R3 npc[5];
  for (int n = 0; n < 5; ++n) npc[n] = {0., 0., 0.};
  for (int n = 0; n < 4; ++n) {
    npc[n + 1].x = 0.5 * (coord[n + 1].y - coord[n].y);
    npc[n + 1].y = 0.5 * (coord[n].x - coord[n + 1].x);
  }
  npc[0] = npc[4];
  for (int ii = 0; ii < 4; ++ii) out[ii] = npc[ii + 1] + npc[ii];
}

// ---------------------------------------------------------------------------
// remap limiters (UtilesRemap.cc:108-120, 329-345)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double flux_limiter(int id, double r) {
  if (id == 0) return smax(0.0, smin(1.0, r));
  if (id == 1) return smax(0.0, smax(smin(2.0 * r, 1.0), smin(r, 2.0)));
  if (id == 2) return (r <= 0.0) ? 0.0 : 2.0 * r / (1.0 + r);
  return 0.0;
}
// x / y with IEEE round-to-nearest, taking the zero-numerator case out of
// the division: 0 / y is exactly +-0 (sign of x xor sign of y) for every y
// other than 0 and NaN, and such quotients (absent materials, flat fields)
// would otherwise leave the division's fast path.
__host__ __device__ __forceinline__ double div_rn(double x, double y) {
#ifdef __CUDA_ARCH__
  if (x == 0.0 && y == y && y != 0.0)
    return ((__double_as_longlong(x) ^ __double_as_longlong(y)) < 0) ? -0.0 : 0.0;
#else
  if (x == 0.0 && y == y && y != 0.0) return std::signbit(x) != std::signbit(y) ? -0.0 : 0.0;
#endif
  return x / y;
}

// limiter id as a template argument: 0-2 the classical limiters (one
// instance each), LIM_ORDER1 a first-order remap (no slope), LIM_GEN the
// generalised limiters 3-7 (id read at run time), LIM_O3 the third-order
// face values of the cell sweep, LIM_PB the pente-borne fluxes of the cell
// sweep (limiter id read at run time)
constexpr int LIM_ORDER1 = 3;
constexpr int LIM_GEN = 4;
constexpr int LIM_O3 = 5;
constexpr int LIM_PB = 6;
// LIM_COLS + (0-2 or LIM_ORDER1): the same cell sweep along y / z with one
// thread per line chunk (body_sweep_cells_cols), for large meshes
constexpr int LIM_COLS = 8;

// RemapADIService::fluxLimiterG (UtilesRemap.cc:130-190): limited slope from
// the back / front gradients gm / gp, the values ym, yp of the neighbours
// and the widths hm, h0, hp of three consecutive cells (or dual cells)
__device__ __forceinline__ double generalized_gradient(int id, double gp, double gm, double yp, double ym,
                                                      double h0, double hp, double hm, int simple_pente) {
  if (gp * gm < 0.0) return 0.;
  const double dy = yp - ym;
  double g = 0.;
  if (id == 3) {
    const double a = smin(fabs(gp), fabs(gm));
    g = dy > 0. ? a : -a;
  } else if (id == 4) {
    const double a = smax(fabs(gp), fabs(gm));
    g = dy > 0. ? a : -a;
  } else if (id == 5) {
    const double lp = (h0 / 2. + hp) / (h0 + hp + hm);
    const double lm = (h0 / 2. + hm) / (h0 + hp + hm);
    const double den = lp * gp + lm * gm;
    g = den != 0. ? gp * gm / den : 0.;
  } else if (id == 7) {
    g = dy / h0;
  } else if (id == 6) {
    const double lp = (h0 / 2. + hp) / (h0 + hp + hm);
    const double lm = (h0 / 2. + hm) / (h0 + hp + hm);
    g = lm * gp + lp * gm;
  }
  if (simple_pente) {
    const double mp = gp * (h0 + hp) / h0;
    const double mm = gm * (h0 + hm) / h0;
    const double a = smin(fabs(smin(fabs(mp), fabs(mm))), fabs(g));
    g = dy > 0. ? a : -a;
  }
  return g;
}
template <int LIM>
__host__ __device__ __forceinline__ double flux_limiter_t(double r) {
  if (LIM == 0) return smax(0.0, smin(1.0, r));
  if (LIM == 1) return smax(0.0, smax(smin(2.0 * r, 1.0), smin(r, 2.0)));
  if (LIM == 2) return (r <= 0.0) ? 0.0 : 2.0 * r / (1.0 + r);
  return 0.0;
}
// computeAndLimitGradPhi (UtilesRemap.cc:325-357):
// g = 0.5 phi(gf / gb) gb + 0.5 phi(gb / gf) gf, each term present when its
// divisor is not zero, phi the flux limiter
template <int LIM>
__host__ __device__ __forceinline__ double limited_gradient_ref(double gb, double gf) {
  double g = 0.;
  if (gb != 0.) g += 0.5 * (flux_limiter_t<LIM>(div_rn(gf, gb)) * gb);
  if (gf != 0.) g += 0.5 * (flux_limiter_t<LIM>(div_rn(gb, gf)) * gf);
  return g;
}

// The same value with one division for minmod and superbee.  With slopes of
// opposite signs, or a zero one, both limiter values are +0 and each term
// is a signed zero, so g = +0.  With same-sign slopes, let n be the slope of
// larger magnitude and d the other: the ratio n / d is >= 1, and comparing
// |n| with |d| and 2 |d| exactly (doubling is exact) tells which branch of
// the limiter the correctly rounded ratios fall in (the bounds 1/2, 1 and 2
// are representable, so rounding never crosses them): minmod gives 1 for
// n / d and d / n itself for the other; superbee gives n / d (<= 2) and 1,
// or 2 and 2 d / n (the ratio < 1/2).  Only the ratio the result depends on
// is divided; the constant term is formed as the reference forms it
// (0.5 (phi x)), so the sum is bit-identical.  Non-finite slopes take the
// reference path.
template <int LIM>
__host__ __device__ __forceinline__ double limited_gradient_t(double gb, double gf) {
  if (LIM != 0 && LIM != 1) return limited_gradient_ref<LIM>(gb, gf);
  const double ab = fabs(gb), af = fabs(gf);
  if (!(ab <= 1.7976931348623157e308 && af <= 1.7976931348623157e308)) return limited_gradient_ref<LIM>(gb, gf);
  if (!((gb > 0. && gf > 0.) || (gb < 0. && gf < 0.))) return 0.;
  const bool fbig = af >= ab;             // the forward slope is n
  const double n = fbig ? gf : gb, d = fbig ? gb : gf;
  double tn, td;                          // terms whose limiter argument is n / d, d / n
  if (LIM == 0) {
    // minmod: phi(n / d) = 1, phi(d / n) = d / n
    tn = 0.5 * (1.0 * d);
    td = 0.5 * (flux_limiter_t<LIM>(div_rn(d, n)) * n);
  } else if (fabs(n) <= 2.0 * fabs(d)) {
    // superbee, n / d in [1, 2]: phi(n / d) = n / d, phi(d / n) = 1
    tn = 0.5 * (flux_limiter_t<LIM>(div_rn(n, d)) * d);
    td = 0.5 * (1.0 * n);
  } else {
    // superbee, n / d > 2: phi(n / d) = 2, phi(d / n) = 2 d / n
    tn = 0.5 * (2.0 * d);
    td = 0.5 * (flux_limiter_t<LIM>(div_rn(d, n)) * n);
  }
  // the reference adds the term of gf / gb (divisor gb) first
  double g = 0.;
  if (fbig) { g += tn; g += td; }
  else { g += td; g += tn; }
  return g;
}
__device__ __forceinline__ double limited_gradient(int id, double gb, double gf) {
  double g = 0.;
  if (gb != 0.) g += 0.5 * (flux_limiter(id, gf / gb) * gb);
  if (gf != 0.) g += 0.5 * (flux_limiter(id, gb / gf) * gf);
  return g;
}

}  // namespace mhc
