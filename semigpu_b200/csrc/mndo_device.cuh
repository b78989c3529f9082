// Device-side MNDO model: element data, pair geometry, the 22 local-frame two-center
// integrals of one atom pair, their rotation into the molecular frame, one-center integrals
// and STO-6G overlaps.  Everything here is FP64 and per atom pair; the kernels decide how
// pairs map onto threads.
//
// Parity notes (reference LuisAlfredoNu/semiGPU, src/common):
//   * element constants: MNDO_parameters.cpp:47-122 (the later dd[7][1], dd[8][1] values win,
//     :95-96, :115-116), STO-6G "Sparrow" sets STO-6G.cpp:42-54, 92-118, 155-181, 219-245;
//   * unit constants: mymath.h:84-97;
//   * the 22 interactions: multipole.cpp:20-492; their combination and the rotation:
//     twocenterintegral.cpp:468-736 (the reference re-derives them for each of the 100
//     elements of a block; here they are derived once per pair and reused);
//   * one-center integrals: twocenterintegral.cpp:738-778;
//   * overlap: overlap.cpp:68-192.  The reference integrates each Cartesian factor with a
//     12-point Gauss-Hermite rule, which is exact for the degree <= 2 polynomials that occur,
//     so the closed forms below agree with it to rounding.
#pragma once
#include <cstdint>

namespace sgb {

constexpr double kAng2Bohr = 1.8897259886;
constexpr double kBohr2Ang = 0.529177249;
constexpr double kHartree2eV = 27.211386;
constexpr double kPi = 3.14159265358979323846;

// Element slot: 0 = H, 1 = C, 2 = N, 3 = O.
struct ElemParams {
  double uss, upp, beta_s, beta_p, alpha, gss, gpp, gsp, gp2, hsp;
  double dd1, dd2;     // charge separations, bohr
  double rho[3];       // Klopman-Ohno additive terms l = 0, 1, 2, bohr
  int core;            // core charge
  int z;
};

struct StoParams {
  double es[6], cs[6], ep[6], cp[6];
};

#ifdef __CUDACC__
__constant__ ElemParams c_elem[4];
__constant__ StoParams c_sto[4];
#endif

// Host copy used to fill the constant bank (defined in mndo_tables.cuh).
extern const ElemParams kElemHost[4];
extern const StoParams kStoHost[4];

// MOPAC pair order SS,SX,XX,SY,XY,YY,SZ,XZ,YZ,ZZ (twocenterintegral.cpp:315-325, 420-421).
__host__ __device__ inline int pair_index(int a, int b) {
  // a, b in 0..3 (s,x,y,z); symmetric
  if (a > b) { int t = a; a = b; b = t; }
  return b * (b + 1) / 2 + a;
}
__host__ __device__ inline int pair_first(int p) {
  // inverse of pair_index: returns the smaller code
  return p == 0 ? 0 : p == 1 ? 0 : p == 2 ? 1 : p == 3 ? 0 : p == 4 ? 1 : p == 5 ? 2 : p == 6 ? 0 : p == 7 ? 1 : p == 8 ? 2 : 3;
}
__host__ __device__ inline int pair_second(int p) {
  return p == 0 ? 0 : p <= 2 ? 1 : p <= 5 ? 2 : 3;
}

#ifdef __CUDACC__

// ------------------------------------------------------------------------------------------
// Local-frame integrals of one pair.  P is the atom of the bra pair, Q of the ket pair; the
// local z axis points from P to Q.  Values are in Hartree.
enum LocalIdx {
  L_SSSS = 0, L_SS_SPZ, L_SPZ_SS, L_SS_PIPI, L_SS_ZZ, L_PIPI_SS, L_ZZ_SS,
  L_SP_SP_PI, L_SP_SP_Z, L_SP_PP_1, L_SP_PP_2, L_SP_PP_3, L_PP_SP_1, L_PP_SP_2, L_PP_SP_3,
  L_ZZZZ, L_PPPP, L_ZZPP, L_PPZZ, L_PZPZ, L_XXYY, L_XYXY, L_COUNT
};

struct PairFrame {
  double v[L_COUNT];
  double rot[9];  // rot[3*k + g]: local axis k (0 = x, 1 = y, 2 = z) along global axis g
};

__device__ __forceinline__ double ko(double scale, double x2) { return 1.0 / (scale * sqrt(x2)); }

struct MultipoleArgs {
  double R, dP1, dP2, dQ1, dQ2;
  double rP[3], rQ[3];
  __device__ __forceinline__ double add(int l, int m) const {
    double s = rP[l] + rQ[m];
    return s * s;
  }
  __device__ __forceinline__ MultipoleArgs swapped() const {
    MultipoleArgs h;
    h.R = R; h.dP1 = dQ1; h.dP2 = dQ2; h.dQ1 = dP1; h.dQ2 = dP2;
    for (int l = 0; l < 3; ++l) { h.rP[l] = rQ[l]; h.rQ[l] = rP[l]; }
    return h;
  }
};

// One function per interaction of multipole.cpp (line of the reference body in brackets).
__device__ __forceinline__ double m_qq(const MultipoleArgs& g) { return ko(1.0, g.R * g.R + g.add(0, 0)); }  // [20]
__device__ inline double m_qUz(const MultipoleArgs& g) {  // [32]
  double a = g.add(0, 1), R = g.R, d = g.dQ1;
  return ko(2.0, (R + d) * (R + d) + a) - ko(2.0, (R - d) * (R - d) + a);
}
__device__ inline double m_qQpipi(const MultipoleArgs& g) {  // [61]
  double a = g.add(0, 2), R = g.R, d = 2.0 * g.dQ2;
  return ko(2.0, R * R + d * d + a) - ko(2.0, R * R + a);
}
__device__ inline double m_qQzz(const MultipoleArgs& g) {  // [89]
  double a = g.add(0, 2), R = g.R, d = 2.0 * g.dQ2;
  return ko(4.0, (R + d) * (R + d) + a) - ko(2.0, R * R + a) + ko(4.0, (R - d) * (R - d) + a);
}
__device__ inline double m_UpiUpi(const MultipoleArgs& g) {  // [123]
  double a = g.add(1, 1), R = g.R, dm = g.dP1 - g.dQ1, dp = g.dP1 + g.dQ1;
  return ko(2.0, R * R + dm * dm + a) - ko(2.0, R * R + dp * dp + a);
}
__device__ inline double m_UzUz(const MultipoleArgs& g) {  // [145]
  double a = g.add(1, 1), R = g.R, s = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double x = (i ? -g.dP1 : g.dP1) + (j ? -g.dQ1 : g.dQ1) + R;
      s += ((i + j) == 1 ? 1.0 : -1.0) * ko(4.0, x * x + a);
    }
  return s;
}
__device__ inline double m_UpiQpiz(const MultipoleArgs& g) {  // [168]
  double a = g.add(1, 2), R = g.R, s = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double x = R + (i ? -g.dQ2 : g.dQ2), y = g.dP1 + (j ? -g.dQ2 : g.dQ2);
      s += ((i + j) == 1 ? 1.0 : -1.0) * ko(4.0, x * x + y * y + a);
    }
  return s;
}
__device__ inline double m_UzQpipi(const MultipoleArgs& g) {  // [199]
  double a = g.add(1, 2), R = g.R, q = 2.0 * g.dQ2, s = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -g.dP1 : g.dP1);
    s += (i ? 1.0 : -1.0) * ko(4.0, x * x + q * q + a);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -g.dP1 : g.dP1);
    s += (i ? -1.0 : 1.0) * ko(4.0, x * x + a);
  }
  return s;
}
__device__ inline double m_UzQz(const MultipoleArgs& g) {  // [233]
  double a = g.add(1, 2), R = g.R, s = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double x = R + (i ? -g.dP1 : g.dP1) + (j ? -2.0 : 2.0) * g.dQ2;
      s += (i ? 1.0 : -1.0) * ko(8.0, x * x + a);
    }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -g.dP1 : g.dP1);
    s += (i ? -1.0 : 1.0) * ko(4.0, x * x + a);
  }
  return s;
}
__device__ inline double m_QpipiQpipi(const MultipoleArgs& g) {  // [270]
  double a = g.add(2, 2), R2 = g.R * g.R, s = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double d = g.dP2 + (i ? -g.dQ2 : g.dQ2);
    s += ko(8.0, R2 + 4.0 * d * d + a);
  }
  double p = 2.0 * g.dP2, q = 2.0 * g.dQ2;
  s -= ko(4.0, R2 + p * p + a);
  s -= ko(4.0, R2 + q * q + a);
  return s + ko(4.0, R2 + a);
}
__device__ inline double m_QxxQyy(const MultipoleArgs& g) {  // [309]
  double a = g.add(2, 2), R2 = g.R * g.R, p = 2.0 * g.dP2, q = 2.0 * g.dQ2;
  return ko(4.0, R2 + p * p + q * q + a) - ko(4.0, R2 + p * p + a) - ko(4.0, R2 + q * q + a) +
         ko(4.0, R2 + a);
}
__device__ inline double m_QpipiQzz(const MultipoleArgs& g) {  // [345]
  double a = g.add(2, 2), R = g.R, p = 2.0 * g.dP2, s = 0.0, aux = p * p + a;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -2.0 : 2.0) * g.dQ2;
    s += ko(8.0, x * x + aux);
    s -= ko(8.0, x * x + a);
    s -= ko(8.0, R * R + aux);
  }
  return s + ko(4.0, R * R + a);
}
__device__ inline double m_QzzQzz(const MultipoleArgs& g) {  // [385]
  double a = g.add(2, 2), R = g.R, s = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double x = R + (i ? -2.0 : 2.0) * g.dP2 + (j ? -2.0 : 2.0) * g.dQ2;
      s += ko(16.0, x * x + a);
    }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -2.0 : 2.0) * g.dP2, y = R + (i ? -2.0 : 2.0) * g.dQ2;
    s -= ko(8.0, x * x + a);
    s -= ko(8.0, y * y + a);
  }
  return s + ko(4.0, R * R + a);
}
__device__ inline double m_QpizQpiz(const MultipoleArgs& g) {  // [425]
  double a = g.add(2, 2), R = g.R, s = 0.0;
  int c = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        // sign pattern +,-,-,+,-,+,+,- over (i,j,k) = parity of i+j+k
        double sg = ((i + j + k) & 1) ? -1.0 : 1.0;
        double x = R + (i ? -g.dP2 : g.dP2) + (j ? -g.dQ2 : g.dQ2);
        double y = g.dP2 + (k ? -g.dQ2 : g.dQ2);
        s += sg * ko(8.0, x * x + y * y + a);
        ++c;
      }
  return s;
}

// Local frame of twocenterintegral.cpp:468-490: z from P to Q; if z is (anti)parallel to the
// global z axis the frame is the global x, y; otherwise y = (-z_y, z_x, 0)/|.|, x = z cross y.
__device__ inline void local_frame(const double* pP, const double* pQ, double R, double* rot) {
#pragma unroll
  for (int c = 0; c < 3; ++c) rot[6 + c] = (pQ[c] - pP[c]) / R;
  if (fabs(rot[6]) < 1e-10 && fabs(rot[7]) < 1e-10) {
    rot[3] = 0.0; rot[4] = 1.0; rot[5] = 0.0;
    rot[0] = 1.0; rot[1] = 0.0; rot[2] = 0.0;
  } else {
    double m = 1.0 / sqrt(rot[6] * rot[6] + rot[7] * rot[7]);
    rot[3] = -m * rot[7];
    rot[4] = m * rot[6];
    rot[5] = 0.0;
    rot[0] = rot[7] * rot[5] - rot[8] * rot[4];
    rot[1] = rot[8] * rot[3] - rot[6] * rot[5];
    rot[2] = rot[6] * rot[4] - rot[7] * rot[3];
  }
}

__device__ __forceinline__ MultipoleArgs multipole_args(int sP, int sQ, double R) {
  MultipoleArgs g;
  g.R = R;
  g.dP1 = c_elem[sP].dd1; g.dP2 = c_elem[sP].dd2;
  g.dQ1 = c_elem[sQ].dd1; g.dQ2 = c_elem[sQ].dd2;
#pragma unroll
  for (int l = 0; l < 3; ++l) { g.rP[l] = c_elem[sP].rho[l]; g.rQ[l] = c_elem[sQ].rho[l]; }
  return g;
}

// All local-frame integrals of one pair.  heavyP / heavyQ select which are needed
// (H-H: ss|ss only; H-X: the ss|* ones; X-X: all 22).
__device__ inline void pair_frame(int sP, int sQ, const double* pP, const double* pQ,
                                  PairFrame& f) {
  double dx = pP[0] - pQ[0], dy = pP[1] - pQ[1], dz = pP[2] - pQ[2];
  double R = sqrt(dx * dx + dy * dy + dz * dz);
  local_frame(pP, pQ, R, f.rot);
  const MultipoleArgs g = multipole_args(sP, sQ, R);
  const double qq = m_qq(g);
  f.v[L_SSSS] = qq;
  const bool hP = sP != 0, hQ = sQ != 0;
  if (hQ) {
    f.v[L_SS_SPZ] = m_qUz(g);
    f.v[L_SS_PIPI] = qq + m_qQpipi(g);
    f.v[L_SS_ZZ] = qq + m_qQzz(g);
  }
  if (hP) {
    const MultipoleArgs h = g.swapped();
    const double Uzq = -m_qUz(h);
    const double Qpipiq = m_qQpipi(h), Qzzq = m_qQzz(h);
    f.v[L_SPZ_SS] = Uzq;
    f.v[L_PIPI_SS] = qq + Qpipiq;
    f.v[L_ZZ_SS] = qq + Qzzq;
    if (hQ) {
      const double qUz = f.v[L_SS_SPZ];
      const double qQpipi = f.v[L_SS_PIPI] - qq, qQzz = f.v[L_SS_ZZ] - qq;
      f.v[L_SP_SP_PI] = m_UpiUpi(g);
      f.v[L_SP_SP_Z] = m_UzUz(g);
      f.v[L_SP_PP_1] = Uzq + m_UzQpipi(g);
      f.v[L_SP_PP_2] = Uzq + m_UzQz(g);
      f.v[L_SP_PP_3] = m_UpiQpiz(g);
      f.v[L_PP_SP_1] = qUz - m_UzQpipi(h);
      f.v[L_PP_SP_2] = qUz - m_UzQz(h);
      f.v[L_PP_SP_3] = -m_UpiQpiz(h);
      const double pppp = qq + qQpipi + Qpipiq + m_QpipiQpipi(g);
      const double xxyy = qq + qQpipi + Qpipiq + m_QxxQyy(g);
      f.v[L_ZZZZ] = qq + qQzz + Qzzq + m_QzzQzz(g);
      f.v[L_PPPP] = pppp;
      f.v[L_ZZPP] = qq + qQpipi + Qzzq + m_QpipiQzz(h);
      f.v[L_PPZZ] = qq + Qpipiq + qQzz + m_QpipiQzz(g);
      f.v[L_PZPZ] = m_QpizQpiz(g);
      f.v[L_XXYY] = xxyy;
      f.v[L_XYXY] = 0.5 * (pppp - xxyy);
    }
  }
}

// (ab|cd) in eV for a, b on P and c, d on Q (angular codes 0..3, a<=b, c<=d), from the
// pair's local integrals: the case split of ComputeTwoCenterIntegral
// (twocenterintegral.cpp:144-227) including the pair-order inversion of CorrectOrderIntegral.
__device__ inline double two_center_value(const PairFrame& f, int a, int b, int c, int d) {
  const double* r = f.rot;
#define RT(k, t) r[3 * (k) + (t)-1]
  const int pa = (a > 0) + (b > 0), pc = (c > 0) + (d > 0);
  double v;
  if (pa == 0) {
    if (pc == 0) {
      v = f.v[L_SSSS];
    } else if (pc == 1) {
      v = f.v[L_SS_SPZ] * RT(2, d);
    } else {
      v = f.v[L_SS_PIPI] * (RT(0, c) * RT(0, d) + RT(1, c) * RT(1, d)) +
          f.v[L_SS_ZZ] * RT(2, c) * RT(2, d);
    }
  } else if (pa == 1) {
    if (pc == 0) {
      v = f.v[L_SPZ_SS] * RT(2, b);
    } else if (pc == 1) {
      v = f.v[L_SP_SP_PI] * (RT(0, b) * RT(0, d) + RT(1, b) * RT(1, d)) +
          f.v[L_SP_SP_Z] * RT(2, b) * RT(2, d);
    } else {
      v = f.v[L_SP_PP_1] * RT(2, b) * (RT(0, c) * RT(0, d) + RT(1, c) * RT(1, d)) +
          f.v[L_SP_PP_2] * RT(2, b) * RT(2, c) * RT(2, d) +
          f.v[L_SP_PP_3] * (RT(0, b) * (RT(2, c) * RT(0, d) + RT(2, d) * RT(0, c)) +
                            RT(1, b) * (RT(2, c) * RT(1, d) + RT(2, d) * RT(1, c)));
    }
  } else {
    if (pc == 0) {
      v = f.v[L_PIPI_SS] * (RT(0, a) * RT(0, b) + RT(1, a) * RT(1, b)) +
          f.v[L_ZZ_SS] * RT(2, a) * RT(2, b);
    } else if (pc == 1) {
      v = f.v[L_PP_SP_1] * RT(2, d) * (RT(0, a) * RT(0, b) + RT(1, a) * RT(1, b)) +
          f.v[L_PP_SP_2] * RT(2, d) * RT(2, a) * RT(2, b) +
          f.v[L_PP_SP_3] * (RT(0, d) * (RT(2, a) * RT(0, b) + RT(2, b) * RT(0, a)) +
                            RT(1, d) * (RT(2, a) * RT(1, b) + RT(2, b) * RT(1, a)));
    } else {
      const double x0a = RT(0, a), x0b = RT(0, b), x0c = RT(0, c), x0d = RT(0, d);
      const double x1a = RT(1, a), x1b = RT(1, b), x1c = RT(1, c), x1d = RT(1, d);
      const double x2a = RT(2, a), x2b = RT(2, b), x2c = RT(2, c), x2d = RT(2, d);
      // pi-z mixing: sum over the (a,b) and (c,d) orderings of x{k}_{first} x2_{second}
      const double m0ab = x0a * x2b + x0b * x2a, m0cd = x0c * x2d + x0d * x2c;
      const double m1ab = x1a * x2b + x1b * x2a, m1cd = x1c * x2d + x1d * x2c;
      const double nab = x0a * x1b + x0b * x1a, ncd = x0c * x1d + x0d * x1c;
      v = f.v[L_ZZZZ] * x2a * x2b * x2c * x2d +
          f.v[L_PPPP] * (x0a * x0b * x0c * x0d + x1a * x1b * x1c * x1d) +
          f.v[L_ZZPP] * x2a * x2b * (x0c * x0d + x1c * x1d) +
          f.v[L_PPZZ] * (x0a * x0b + x1a * x1b) * x2c * x2d +
          f.v[L_PZPZ] * (m0ab * m0cd + m1ab * m1cd) +
          f.v[L_XXYY] * (x0a * x0b * x1c * x1d + x1a * x1b * x0c * x0d) +
          f.v[L_XYXY] * nab * ncd;
    }
  }
#undef RT
  return v * kHartree2eV;
}

// One-center (ab|cd) on an atom, eV (twocenterintegral.cpp:738-778).
__device__ __forceinline__ double one_center_value(int slot, int a, int b, int c, int d) {
  const ElemParams& e = c_elem[slot];
  const int p1 = (a > 0) + (b > 0), p2 = (c > 0) + (d > 0);
  if (p1 == p2) {
    if (p1 == 0) return e.gss;
    if (p1 == 1) return b == d ? e.hsp : 0.0;
    if (a == b && c == d) return a == c ? e.gpp : e.gp2;
    if (a == c && b == d) return 0.5 * (e.gpp - e.gp2);
    return 0.0;
  }
  if (p1 == 0 && p2 == 2) return c == d ? e.gsp : 0.0;
  if (p1 == 2 && p2 == 0) return a == b ? e.gsp : 0.0;
  return 0.0;
}

// STO-6G overlap block between atoms A (bra) and B (ket), S[4*mu + nu], mu over A's AOs
// (s, px, py, pz) and nu over B's.  Only the first nA x nB entries are meaningful.
__device__ inline void overlap_block(int sA, int sB, const double* pA, const double* pB,
                                     double* S) {
  const double ab[3] = {pB[0] - pA[0], pB[1] - pA[1], pB[2] - pA[2]};
  const double r2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
  const bool hA = sA != 0, hB = sB != 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) S[k] = 0.0;
  const StoParams& ta = c_sto[sA];
  const StoParams& tb = c_sto[sB];
  // shell combos: (s,s), (s,p), (p,s), (p,p)
  for (int combo = 0; combo < 4; ++combo) {
    const bool pa = combo & 2, pb = combo & 1;
    if ((pa && !hA) || (pb && !hB)) continue;
    const double* ea = pa ? ta.ep : ta.es;
    const double* ca = pa ? ta.cp : ta.cs;
    const double* eb = pb ? tb.ep : tb.es;
    const double* cb = pb ? tb.cp : tb.cs;
    double acc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = 0.0;
    for (int i = 0; i < 6; ++i) {
      for (int j = 0; j < 6; ++j) {
        const double al = ea[i], be = eb[j], p = al + be, ip = 1.0 / p;
        const double sq = sqrt(kPi * ip);
        const double K = exp(-al * be * ip * r2) * ca[i] * cb[j] * sq * sq * sq;
        if (!pa && !pb) {
          acc[0] += K;
        } else if (!pa && pb) {  // P - B = al/p * (A - B) = -al/p * ab
#pragma unroll
          for (int t = 0; t < 3; ++t) acc[t] += K * (-al * ip * ab[t]);
        } else if (pa && !pb) {  // P - A = be/p * ab
#pragma unroll
          for (int t = 0; t < 3; ++t) acc[t] += K * (be * ip * ab[t]);
        } else {
#pragma unroll
          for (int t = 0; t < 3; ++t)
#pragma unroll
            for (int u = 0; u < 3; ++u)
              acc[3 * t + u] += K * ((be * ip * ab[t]) * (-al * ip * ab[u]) + (t == u ? 0.5 * ip : 0.0));
        }
      }
    }
    if (!pa && !pb) {
      S[0] = acc[0];
    } else if (!pa && pb) {
      for (int t = 0; t < 3; ++t) S[1 + t] = acc[t];
    } else if (pa && !pb) {
      for (int t = 0; t < 3; ++t) S[4 * (1 + t)] = acc[t];
    } else {
      for (int t = 0; t < 3; ++t)
        for (int u = 0; u < 3; ++u) S[4 * (1 + t) + 1 + u] = acc[3 * t + u];
    }
  }
}

#endif  // __CUDACC__

}  // namespace sgb
