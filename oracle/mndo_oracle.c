/* TEST INFRASTRUCTURE ONLY — the CPU oracle for the MNDO hot path.
 *
 * A plain-C restatement of the reference's algorithm (LuisAlfredoNu/semiGPU, src/common) used
 * by the parity tests, by the test-side checks in __graft_entry__.smoke() and by bench.py's
 * cpu_baseline leg.  It is never linked into, loaded by, or called from the product library.
 * Its outputs are pinned against golden vectors produced by the unmodified reference build
 * (oracle/_ref/ref_driver, fixtures under tests/golden/).
 *
 * Conventions (all follow the reference):
 *   - atoms in input order; an H atom owns one AO (s), C/N/O own four (s, px, py, pz)
 *     (atomicOrbitals.cpp:76-119); angular code 0=s 1=x 2=y 3=z (atomicOrbitals.cpp:23-31)
 *   - coordinates enter in Angstrom and are converted to bohr with 1.8897259886 (mymath.h:84-87)
 *   - matrices are packed lower triangles, index i*(i+1)/2+j for i>=j (mymemory.cpp:369-371)
 *   - integral storage is the reference's ragged [A][B<=A] array flattened in that order:
 *     X-X pairs 10x10, H-X / X-H pairs 1x10, H-H pairs 1x1, row-major
 *     (twocenterintegral.cpp:55-107); pair index order SS,SX,XX,SY,XY,YY,SZ,XZ,YZ,ZZ
 *     (twocenterintegral.cpp:315-325, 420-421).
 */
#define _DEFAULT_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ANG2BOHR 1.8897259886 /* mymath.h:86 */
#define BOHR2ANG 0.529177249  /* mymath.h:91 */
#define HA2EV 27.211386       /* mymath.h:96 */

/* ---------------------------------------------------------------------------------------- */
/* Element data: MNDO_parameters.cpp:47-122 (effective values: the later dd[7][1], dd[8][1]
 * assignments win, :95-96 and :115-116) and the "Sparrow" STO-6G sets that overwrite the
 * earlier ones in STO-6G.cpp (H :42-54, C :92-118, N :155-181, O :219-245). Index by Z. */
typedef struct {
  double uss, upp, beta_s, beta_p, alpha, gss, gpp, gsp, gp2, hsp, dd1, dd2, pp0, pp1, pp2;
} elem_t;

static const elem_t ELEM[9] = {
    [1] = {-11.90627600, 0.0, -6.98906400, 0.0, 2.54413410, 12.848, 0.0, 0.0, 0.0, 0.0, 0.0,
           0.0, 1.05897351, 0.0, 0.0},
    [6] = {-52.27974500, -39.20555800, -18.9850440, -7.93412200, 2.546380, 12.23, 11.08, 11.47,
           9.84, 2.43, 0.80746618, 0.68515777, 1.11248501, 0.81309641, 0.74785493},
    [7] = {-71.93212200, -57.17231900, -20.49575800, -20.49575800, 2.86134200, 13.59, 12.98,
           12.66, 11.59, 3.14, 0.63990367, 0.54297627, 1.00115465, 0.63747362, 0.61528499},
    [8] = {-99.64430900, -77.79747200, -32.68808200, -32.68808200, 3.16060400, 15.42, 14.52,
           14.48, 12.98, 3.94, 0.53460239, 0.45362517, 0.88234058, 0.52124931, 0.52654944},
};

typedef struct {
  double es[6], cs[6], ep[6], cp[6];
} sto_t;

static const sto_t STO[9] = {
    [1] = {{4.098792193376860e+01, 7.515090619202102e+00, 2.102451537968084e+00,
            7.222488471249888e-01, 2.804703624957924e-01, 1.155131838418812e-01},
           {1.057956874127020e-01, 1.596794562489045e-01, 2.097264517638662e-01,
            2.069126553471125e-01, 1.144014417359658e-01, 1.840525175585220e-02},
           {0},
           {0}},
    [6] = {{8.846144274163005e+01, 1.622292919221501e+01, 4.558993095148346e+00,
            6.519461344814428e-01, 2.958932522507792e-01, 1.411098199523801e-01},
           {-8.534093658582062e-02, -1.190837759635380e-01, -1.145234971659361e-01,
            1.730334274890658e-01, 1.607236215755646e-01, 2.810826497961667e-02},
           {1.875086664726173e+01, 4.889844711496806e+00, 1.749633028685196e+00,
            7.313800499385337e-01, 3.344367808801327e-01, 1.581099099775126e-01},
           {4.407314493338078e-01, 5.331737162464377e-01, 5.445171182695406e-01,
            3.904445162839797e-01, 1.454563993779586e-01, 1.494840672526637e-02}},
    [7] = {{1.408553999528384e+02, 2.583144824406823e+01, 7.259194242116380e+00,
            1.038080893483724e+00, 4.711449542017903e-01, 2.246863662931398e-01},
           {-1.209684224448265e-01, -1.687979660569579e-01, -1.623338967119989e-01,
            2.452701082384343e-01, 2.278212980714544e-01, 3.984268990094886e-02},
           {2.985663289232627e+01, 7.786002705798312e+00, 2.785905953918744e+00,
            1.164561940873007e+00, 5.325170500259336e-01, 2.517552723103985e-01},
           {7.883124678886093e-01, 9.536589428843584e-01, 9.739482715823707e-01,
            6.983669549124415e-01, 2.601699818271488e-01, 2.673740531657013e-02}},
    [8] = {{2.018091738330405e+02, 3.700975064350955e+01, 1.040053837613310e+01,
            1.487300079059505e+00, 6.750282487920551e-01, 3.219171573709536e-01},
           {-1.584154624760238e-01, -2.210511414259479e-01, -2.125860518260085e-01,
            3.211960348235300e-01, 2.983457630220672e-01, 5.217641116074215e-02},
           {4.277679392805792e+01, 1.115531796470053e+01, 3.991479056714438e+00,
            1.668514542173559e+00, 7.629585088943974e-01, 3.606998633356254e-01},
           {1.235684643746845e+00, 1.494866260646997e+00, 1.526669908217376e+00,
            1.094694498739664e+00, 4.078180472887439e-01, 4.191104734371579e-02}},
};

static int supported(int z) { return z == 1 || z == 6 || z == 7 || z == 8; }
/* atomicOrbitals.cpp:46-64 */
static int core_charge(int z) { return z < 2 ? z : z - 2; }
static int nao_of(int z) { return z < 2 ? 1 : 4; }

/* pair index of two angular codes (a<=b after sorting), twocenterintegral.cpp:315-325 */
static int pair_index(int a, int b) {
  static const int tab[4][4] = {{0, 1, 3, 6}, {1, 2, 4, 7}, {3, 4, 5, 8}, {6, 7, 8, 9}};
  return tab[a][b];
}
/* MOPAC pair order, twocenterintegral.cpp:420-421 */
static const int PAIR_A[10] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3};
static const int PAIR_B[10] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3};

/* ---------------------------------------------------------------------------------------- */
/* Molecule bookkeeping */
typedef struct {
  int natoms, nao;
  const int *Z;
  double *pos;      /* bohr, 3*natoms */
  int *first;       /* first AO of each atom */
  long *blk_off;    /* offset of block [A][B] (B<=A) in the ragged storage, index A*(A+1)/2+B */
  long blk_total;
} mol_t;

static long tri(long i) { return i * (i + 1) / 2; }

static int block_rows(int za, int zb) { return (za > 1 && zb > 1) ? 10 : 1; }
static int block_cols(int za, int zb) { return (za == 1 && zb == 1) ? 1 : 10; }

static int mol_init(mol_t *m, int natoms, const int *Z, const double *xyz_ang) {
  memset(m, 0, sizeof(*m));
  if (natoms <= 0) return -1;
  for (int a = 0; a < natoms; ++a)
    if (!supported(Z[a])) return -2;
  m->natoms = natoms;
  m->Z = Z;
  m->pos = (double *)malloc(sizeof(double) * 3 * natoms);
  m->first = (int *)malloc(sizeof(int) * natoms);
  m->blk_off = (long *)malloc(sizeof(long) * tri(natoms));
  int k = 0;
  for (int a = 0; a < natoms; ++a) {
    m->first[a] = k;
    k += nao_of(Z[a]);
    for (int c = 0; c < 3; ++c) m->pos[3 * a + c] = xyz_ang[3 * a + c] * ANG2BOHR;
  }
  m->nao = k;
  long off = 0;
  for (int a = 0; a < natoms; ++a)
    for (int b = 0; b <= a; ++b) {
      m->blk_off[tri(a) + b] = off;
      off += block_rows(Z[a], Z[b]) * block_cols(Z[a], Z[b]);
    }
  m->blk_total = off;
  return 0;
}

static void mol_free(mol_t *m) {
  free(m->pos);
  free(m->first);
  free(m->blk_off);
}

static double dist(const double *a, const double *b) {
  double r = 0.0;
  for (int c = 0; c < 3; ++c) r += (a[c] - b[c]) * (a[c] - b[c]);
  return sqrt(r);
}

/* ---------------------------------------------------------------------------------------- */
/* Klopman-Ohno multipole-multipole interactions in the local frame (Hartree), one function
 * per interaction of multipole.cpp:20-492.  P is the atom of the first charge distribution,
 * Q the second; R in bohr.  add(l,m) = (rho_P[l] + rho_Q[m])^2 (multipole.cpp:494-498). */
typedef struct {
  double R, dP1, dP2, dQ1, dQ2;
  double rP[3], rQ[3];
} pairgeom_t;

static double add_(const pairgeom_t *g, int l, int m) {
  double s = g->rP[l] + g->rQ[m];
  return s * s;
}
static double inv(double scale, double x2) { return 1.0 / (scale * sqrt(x2)); }

static pairgeom_t swapped(const pairgeom_t *g) {
  pairgeom_t h = *g;
  h.dP1 = g->dQ1; h.dP2 = g->dQ2; h.dQ1 = g->dP1; h.dQ2 = g->dP2;
  for (int l = 0; l < 3; ++l) { h.rP[l] = g->rQ[l]; h.rQ[l] = g->rP[l]; }
  return h;
}

static double m_qq(const pairgeom_t *g) { return inv(1.0, g->R * g->R + add_(g, 0, 0)); } /* :20 */
static double m_qUz(const pairgeom_t *g) {                                                   /* :32 */
  double a = add_(g, 0, 1), R = g->R, d = g->dQ1;
  return inv(2.0, (R + d) * (R + d) + a) - inv(2.0, (R - d) * (R - d) + a);
}
static double m_Uzq(const pairgeom_t *g) { pairgeom_t h = swapped(g); return -m_qUz(&h); } /* :55 */
static double m_qQpipi(const pairgeom_t *g) {                                               /* :61 */
  double a = add_(g, 0, 2), R = g->R, d = 2.0 * g->dQ2;
  return inv(2.0, R * R + d * d + a) - inv(2.0, R * R + a);
}
static double m_Qpipiq(const pairgeom_t *g) { pairgeom_t h = swapped(g); return m_qQpipi(&h); }
static double m_qQzz(const pairgeom_t *g) {                                                 /* :89 */
  double a = add_(g, 0, 2), R = g->R, d = 2.0 * g->dQ2;
  return inv(4.0, (R + d) * (R + d) + a) - inv(2.0, R * R + a) + inv(4.0, (R - d) * (R - d) + a);
}
static double m_Qzzq(const pairgeom_t *g) { pairgeom_t h = swapped(g); return m_qQzz(&h); }
static double m_UpiUpi(const pairgeom_t *g) {                                               /* :123 */
  double a = add_(g, 1, 1), R = g->R, dm = g->dP1 - g->dQ1, dp = g->dP1 + g->dQ1;
  return inv(2.0, R * R + dm * dm + a) - inv(2.0, R * R + dp * dp + a);
}
static double m_UzUz(const pairgeom_t *g) {                                                 /* :145 */
  double a = add_(g, 1, 1), R = g->R, s = 0.0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      double x = (i ? -g->dP1 : g->dP1) + (j ? -g->dQ1 : g->dQ1) + R;
      s += ((i + j) == 1 ? 1.0 : -1.0) * inv(4.0, x * x + a);
    }
  return s;
}
static double m_UpiQpiz(const pairgeom_t *g) {                                              /* :168 */
  double a = add_(g, 1, 2), R = g->R, s = 0.0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      double x = R + (i ? -g->dQ2 : g->dQ2), y = g->dP1 + (j ? -g->dQ2 : g->dQ2);
      s += ((i + j) == 1 ? 1.0 : -1.0) * inv(4.0, x * x + y * y + a);
    }
  return s;
}
static double m_QpizUpi(const pairgeom_t *g) { pairgeom_t h = swapped(g); return -m_UpiQpiz(&h); }
static double m_UzQpipi(const pairgeom_t *g) {                                              /* :199 */
  double a = add_(g, 1, 2), R = g->R, q = 2.0 * g->dQ2, s = 0.0;
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -g->dP1 : g->dP1);
    s += (i ? 1.0 : -1.0) * inv(4.0, x * x + q * q + a);
  }
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -g->dP1 : g->dP1);
    s += (i ? -1.0 : 1.0) * inv(4.0, x * x + a);
  }
  return s;
}
static double m_QpipiUz(const pairgeom_t *g) { pairgeom_t h = swapped(g); return -m_UzQpipi(&h); }
static double m_UzQz(const pairgeom_t *g) {                                                 /* :233 */
  double a = add_(g, 1, 2), R = g->R, s = 0.0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      double x = R + (i ? -g->dP1 : g->dP1) + (j ? -2.0 : 2.0) * g->dQ2;
      s += (i ? 1.0 : -1.0) * inv(8.0, x * x + a);
    }
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -g->dP1 : g->dP1);
    s += (i ? -1.0 : 1.0) * inv(4.0, x * x + a);
  }
  return s;
}
static double m_QzUz(const pairgeom_t *g) { pairgeom_t h = swapped(g); return -m_UzQz(&h); }
static double m_QpipiQpipi(const pairgeom_t *g) {                                           /* :270 */
  double a = add_(g, 2, 2), R2 = g->R * g->R, s = 0.0;
  for (int i = 0; i < 2; ++i) {
    double d = g->dP2 + (i ? -g->dQ2 : g->dQ2);
    s += inv(8.0, R2 + 4.0 * d * d + a);
  }
  double p = 2.0 * g->dP2, q = 2.0 * g->dQ2;
  s -= inv(4.0, R2 + p * p + a);
  s -= inv(4.0, R2 + q * q + a);
  s += inv(4.0, R2 + a);
  return s;
}
static double m_QxxQyy(const pairgeom_t *g) {                                               /* :309 */
  double a = add_(g, 2, 2), R2 = g->R * g->R, p = 2.0 * g->dP2, q = 2.0 * g->dQ2;
  return inv(4.0, R2 + p * p + q * q + a) - inv(4.0, R2 + p * p + a) - inv(4.0, R2 + q * q + a) +
         inv(4.0, R2 + a);
}
static double m_QpipiQzz(const pairgeom_t *g) {                                             /* :345 */
  double a = add_(g, 2, 2), R = g->R, p = 2.0 * g->dP2, s = 0.0;
  double aux = p * p + a;
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -2.0 : 2.0) * g->dQ2;
    s += inv(8.0, x * x + aux);
    s -= inv(8.0, x * x + a);
    s -= inv(8.0, R * R + aux);
  }
  return s + inv(4.0, R * R + a);
}
static double m_QzzQpipi(const pairgeom_t *g) { pairgeom_t h = swapped(g); return m_QpipiQzz(&h); }
static double m_QzzQzz(const pairgeom_t *g) {                                               /* :385 */
  double a = add_(g, 2, 2), R = g->R, s = 0.0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      double x = R + (i ? -2.0 : 2.0) * g->dP2 + (j ? -2.0 : 2.0) * g->dQ2;
      s += inv(16.0, x * x + a);
    }
  for (int i = 0; i < 2; ++i) {
    double x = R + (i ? -2.0 : 2.0) * g->dP2, y = R + (i ? -2.0 : 2.0) * g->dQ2;
    s -= inv(8.0, x * x + a);
    s -= inv(8.0, y * y + a);
  }
  return s + inv(4.0, R * R + a);
}
static double m_QpizQpiz(const pairgeom_t *g) {                                             /* :425 */
  static const double sg[8] = {1, -1, -1, 1, -1, 1, 1, -1};
  double a = add_(g, 2, 2), R = g->R, s = 0.0;
  int c = 0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k) {
        double x = R + (i ? -g->dP2 : g->dP2) + (j ? -g->dQ2 : g->dQ2);
        double y = g->dP2 + (k ? -g->dQ2 : g->dQ2);
        s += sg[c++] * inv(8.0, x * x + y * y + a);
      }
  return s;
}

/* Local frame: z from the first atom to the second; x, y as twocenterintegral.cpp:468-490 */
static void local_frame(const double *pa, const double *pb, double rot[3][3]) {
  double R = dist(pa, pb);
  for (int c = 0; c < 3; ++c) rot[2][c] = (pb[c] - pa[c]) / R;
  if (fabs(rot[2][0]) < 1e-10 && fabs(rot[2][1]) < 1e-10) {
    rot[1][0] = 0.0; rot[1][1] = 1.0; rot[1][2] = 0.0;
    rot[0][0] = 1.0; rot[0][1] = 0.0; rot[0][2] = 0.0;
  } else {
    double m = 1.0 / sqrt(rot[2][0] * rot[2][0] + rot[2][1] * rot[2][1]);
    rot[1][0] = -m * rot[2][1];
    rot[1][1] = m * rot[2][0];
    rot[1][2] = 0.0;
    rot[0][0] = rot[2][1] * rot[1][2] - rot[2][2] * rot[1][1];
    rot[0][1] = rot[2][2] * rot[1][0] - rot[2][0] * rot[1][2];
    rot[0][2] = rot[2][0] * rot[1][1] - rot[2][1] * rot[1][0];
  }
}

/* One two-center element (ab|cd), a,b on atom P and c,d on atom Q != P, angular codes with
 * a<=b, c<=d as the reference stores them; result in eV.  Follows ComputeTwoCenterIntegral
 * (twocenterintegral.cpp:144-227) and IntegralType* (:515-736), including the pair-order
 * inversion of CorrectOrderIntegral (:785-797), which keeps the atom order but swaps which
 * multipole formula is used. */
static double two_center_element(const mol_t *m, int P, int Q, int t0, int t1, int t2, int t3) {
  int zP = m->Z[P], zQ = m->Z[Q];
  pairgeom_t g;
  g.R = dist(m->pos + 3 * P, m->pos + 3 * Q);
  g.dP1 = ELEM[zP].dd1; g.dP2 = ELEM[zP].dd2; g.dQ1 = ELEM[zQ].dd1; g.dQ2 = ELEM[zQ].dd2;
  g.rP[0] = ELEM[zP].pp0; g.rP[1] = ELEM[zP].pp1; g.rP[2] = ELEM[zP].pp2;
  g.rQ[0] = ELEM[zQ].pp0; g.rQ[1] = ELEM[zQ].pp1; g.rQ[2] = ELEM[zQ].pp2;
  int ty[4] = {t0, t1, t2, t3};
  int ptA = (t0 > 0) + (t1 > 0), ptB = (t2 > 0) + (t3 > 0);
  int inverted = 0;
  if (ptA > ptB) {
    int t;
    t = ptA; ptA = ptB; ptB = t;
    t = ty[0]; ty[0] = ty[2]; ty[2] = t;
    t = ty[1]; ty[1] = ty[3]; ty[3] = t;
    inverted = 1;
  }
  double rot[3][3];
  local_frame(m->pos + 3 * P, m->pos + 3 * Q, rot);
#define RT(k, t) rot[k][(t)-1]
  double v = 0.0;
  if (ptA == 0 && ptB == 0) {
    v = m_qq(&g);
  } else if (ptA == 0 && ptB == 1) { /* :520-533 */
    v = (inverted ? m_Uzq(&g) : m_qUz(&g)) * RT(2, ty[3]);
  } else if (ptA == 0 && ptB == 2) { /* :535-559 */
    double qq = m_qq(&g);
    double vpi = qq + (inverted ? m_Qpipiq(&g) : m_qQpipi(&g));
    double vz = qq + (inverted ? m_Qzzq(&g) : m_qQzz(&g));
    v = vpi * RT(0, ty[2]) * RT(0, ty[3]) + vpi * RT(1, ty[2]) * RT(1, ty[3]) +
        vz * RT(2, ty[2]) * RT(2, ty[3]);
  } else if (ptA == 1 && ptB == 1) { /* :561-576 */
    double vpi = m_UpiUpi(&g), vz = m_UzUz(&g);
    v = vpi * RT(0, ty[1]) * RT(0, ty[3]) + vpi * RT(1, ty[1]) * RT(1, ty[3]) +
        vz * RT(2, ty[1]) * RT(2, ty[3]);
  } else if (ptA == 1 && ptB == 2) { /* :578-632 */
    double u, v1, v2, v3;
    if (!inverted) {
      u = m_Uzq(&g);
      v1 = u + m_UzQpipi(&g);
      v2 = u + m_UzQz(&g);
      v3 = m_UpiQpiz(&g);
    } else {
      u = m_qUz(&g);
      v1 = u + m_QpipiUz(&g);
      v2 = u + m_QzUz(&g);
      v3 = m_QpizUpi(&g);
    }
    int b = ty[1], c = ty[2], d = ty[3];
    v = v1 * RT(2, b) * RT(0, c) * RT(0, d) + v1 * RT(2, b) * RT(1, c) * RT(1, d) +
        v2 * RT(2, b) * RT(2, c) * RT(2, d) + v3 * RT(0, b) * RT(2, c) * RT(0, d) +
        v3 * RT(1, b) * RT(2, c) * RT(1, d) + v3 * RT(0, b) * RT(2, d) * RT(0, c) +
        v3 * RT(1, b) * RT(2, d) * RT(1, c);
  } else { /* PP|PP, :634-736 */
    int a = ty[0], b = ty[1], c = ty[2], d = ty[3];
    double qq = m_qq(&g), qQzz = m_qQzz(&g), Qzzq = m_Qzzq(&g);
    double qQpp = m_qQpipi(&g), Qppq = m_Qpipiq(&g);
    double zzzz = qq + qQzz + Qzzq + m_QzzQzz(&g);
    double pppp = qq + qQpp + Qppq + m_QpipiQpipi(&g);
    double zzpp = qq + qQpp + Qzzq + m_QzzQpipi(&g);
    double ppzz = qq + Qppq + qQzz + m_QpipiQzz(&g);
    double pzpz = m_QpizQpiz(&g);
    double xxyy = qq + qQpp + Qppq + m_QxxQyy(&g);
    double xyxy = 0.5 * (pppp - xxyy);
#define R4(i, j, k, l, A, B, C, D) (RT(i, A) * RT(j, B) * RT(k, C) * RT(l, D))
    v = zzzz * R4(2, 2, 2, 2, a, b, c, d) +
        pppp * (R4(0, 0, 0, 0, a, b, c, d) + R4(1, 1, 1, 1, a, b, c, d)) +
        zzpp * (R4(2, 2, 0, 0, a, b, c, d) + R4(2, 2, 1, 1, a, b, c, d)) +
        ppzz * (R4(0, 0, 2, 2, a, b, c, d) + R4(1, 1, 2, 2, a, b, c, d)) +
        pzpz * (R4(0, 2, 0, 2, a, b, c, d) + R4(0, 2, 0, 2, a, b, d, c) + R4(0, 2, 0, 2, b, a, c, d) +
                R4(0, 2, 0, 2, b, a, d, c) + R4(1, 2, 1, 2, a, b, c, d) + R4(1, 2, 1, 2, a, b, d, c) +
                R4(1, 2, 1, 2, b, a, c, d) + R4(1, 2, 1, 2, b, a, d, c)) +
        xxyy * (R4(0, 0, 1, 1, a, b, c, d) + R4(1, 1, 0, 0, a, b, c, d)) +
        xyxy * (R4(0, 1, 0, 1, a, b, c, d) + R4(0, 1, 0, 1, a, b, d, c) + R4(0, 1, 0, 1, b, a, c, d) +
                R4(0, 1, 0, 1, b, a, d, c));
#undef R4
  }
#undef RT
  return v * HA2EV;
}

/* One-center element (ab|cd) on one atom, eV, SelfIntegralType* (twocenterintegral.cpp:738-778) */
static double one_center_element(int z, int a, int b, int c, int d) {
  const elem_t *e = &ELEM[z];
  int p1 = (a > 0) + (b > 0), p2 = (c > 0) + (d > 0);
  if (p1 == p2) {
    if (p1 == 0) return e->gss;
    if (p1 == 1) return b == d ? e->hsp : 0.0;
    if (a == b && c == d) return a == c ? e->gpp : e->gp2;
    if (a == c && b == d) return 0.5 * (e->gpp - e->gp2);
    return 0.0;
  }
  if (p1 == 0 && p2 == 2) return c == d ? e->gsp : 0.0;
  if (p1 == 2 && p2 == 0) return a == b ? e->gsp : 0.0;
  return 0.0;
}

/* Fill every pair block, ComputeAllTwoCenterIntegral + ComputePair_* (twocenterintegral.cpp:
 * 229-279, 388-466): X-X blocks hold (pair on A | pair on B) with A the higher atom index,
 * H-X and X-H blocks hold (s_H s_H | pair on X) computed with the H atom first. */
static void fill_blocks(const mol_t *m, double *blocks) {
  for (int A = 0; A < m->natoms; ++A)
    for (int B = 0; B <= A; ++B) {
      double *blk = blocks + m->blk_off[tri(A) + B];
      int zA = m->Z[A], zB = m->Z[B];
      if (A == B) {
        if (zA == 1) {
          blk[0] = ELEM[1].gss;
        } else {
          for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j)
              blk[10 * i + j] =
                  one_center_element(zA, PAIR_A[i], PAIR_B[i], PAIR_A[j], PAIR_B[j]);
        }
      } else if (zA == 1 && zB == 1) {
        blk[0] = two_center_element(m, A, B, 0, 0, 0, 0);
      } else if (zA > 1 && zB > 1) {
        for (int i = 0; i < 10; ++i)
          for (int j = 0; j < 10; ++j)
            blk[10 * i + j] =
                two_center_element(m, A, B, PAIR_A[i], PAIR_B[i], PAIR_A[j], PAIR_B[j]);
      } else {
        int H = (zA == 1) ? A : B, X = (zA == 1) ? B : A;
        for (int k = 0; k < 10; ++k)
          blk[k] = two_center_element(m, H, X, 0, 0, PAIR_A[k], PAIR_B[k]);
      }
    }
}

/* (mu nu | lam sig) for AOs given by atom and angular code: GetValueFromArray
 * (twocenterintegral.cpp:285-386). Zero unless mu,nu share an atom and lam,sig share one. */
static double eri(const mol_t *m, const double *blocks, int Amu, int tmu, int Anu, int tnu,
                  int Alam, int tlam, int Asig, int tsig) {
  if (Amu != Anu || Alam != Asig) return 0.0;
  int A = Amu, C = Alam, ta = tmu, tb = tnu, tc = tlam, td = tsig;
  if (A < C) {
    int t;
    t = A; A = C; C = t;
    t = ta; ta = tc; tc = t;
    t = tb; tb = td; td = t;
  }
  const double *blk = blocks + m->blk_off[tri(A) + C];
  int zA = m->Z[A], zC = m->Z[C];
  if (zA > 1 && zC > 1) {
    int p = ta <= tb ? pair_index(ta, tb) : pair_index(tb, ta);
    int q = tc <= td ? pair_index(tc, td) : pair_index(td, tc);
    return blk[10 * p + q];
  }
  if (zA == 1 && zC == 1) return blk[0];
  /* mixed: the X side's pair selects the column */
  if (zA > 1) return blk[ta <= tb ? pair_index(ta, tb) : pair_index(tb, ta)];
  return blk[tc <= td ? pair_index(tc, td) : pair_index(td, tc)];
}

typedef struct {
  int atom, ang;
} ao_t;

static ao_t *ao_table(const mol_t *m) {
  ao_t *t = (ao_t *)malloc(sizeof(ao_t) * m->nao);
  for (int A = 0; A < m->natoms; ++A)
    for (int k = 0; k < nao_of(m->Z[A]); ++k) {
      t[m->first[A] + k].atom = A;
      t[m->first[A] + k].ang = k;
    }
  return t;
}

/* ---------------------------------------------------------------------------------------- */
/* STO-6G overlap, Overlap::ComputeOverlap + OverlapNumericalIntegral (overlap.cpp:68-134,
 * 177-192): 6x6 primitives, per-axis 12-point Gauss-Hermite quadrature (nodes/weights of the
 * standard rule, overlap.cpp:47-58). */
static const double GH_X[12] = {-3.889724897869781919272, -3.020637025120889771711,
                                -2.279507080501059900188, -1.59768263515260479671,
                                -0.9477883912401637437046, -0.314240376254359111277,
                                3.889724897869781919272,  3.020637025120889771711,
                                2.279507080501059900188,  1.59768263515260479671,
                                0.9477883912401637437046, 0.314240376254359111277};
static const double GH_W[12] = {2.65855168435630160602E-7, 8.5736870435878586546E-5,
                                0.00390539058462906185999, 0.05160798561588392999187,
                                0.2604923102641611292334,  0.5701352362624795783471,
                                2.65855168435630160602E-7, 8.5736870435878586546E-5,
                                0.00390539058462906185999, 0.05160798561588392999187,
                                0.2604923102641611292334,  0.5701352362624795783471};

static double axis_overlap(int la, int lb, double p, double xa, double xb) {
  double sp = sqrt(p);
  if (la == 0 && lb == 0) return sqrt(M_PI) / sp;
  double s = 0.0;
  for (int i = 0; i < 12; ++i) {
    double x = GH_X[i] / sp;
    s += GH_W[i] * (la ? x + xa : 1.0) * (lb ? x + xb : 1.0);
  }
  return s / sp;
}

static double sto_overlap(int za, int ta, const double *pa, int zb, int tb, const double *pb) {
  double ab2 = 0.0;
  for (int c = 0; c < 3; ++c) ab2 += (pa[c] - pb[c]) * (pa[c] - pb[c]);
  const double *ea = ta ? STO[za].ep : STO[za].es, *ca = ta ? STO[za].cp : STO[za].cs;
  const double *eb = tb ? STO[zb].ep : STO[zb].es, *cb = tb ? STO[zb].cp : STO[zb].cs;
  double s = 0.0;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double al = ea[i], be = eb[j], p = al + be, mu = al * be / p;
      double t = exp(-mu * ab2) * ca[i] * cb[j];
      for (int c = 0; c < 3; ++c) {
        double P = (al * pa[c] + be * pb[c]) / p;
        t *= axis_overlap(ta == c + 1, tb == c + 1, p, P - pa[c], P - pb[c]);
      }
      s += t;
    }
  return s;
}

/* ---------------------------------------------------------------------------------------- */
/* Hcore, Hcore::ComputeElementMatrix and helpers (hcore.cpp:25-100) */
static void build_hcore(const mol_t *m, const ao_t *ao, const double *blocks, double *H) {
  for (int i = 0; i < m->nao; ++i)
    for (int j = 0; j <= i; ++j) {
      int A = ao[i].atom, B = ao[j].atom, zA = m->Z[A], zB = m->Z[B];
      double h;
      if (A == B) {
        double s = 0.0; /* Σ_{C != A} -Z_C (ij | s_C s_C), hcore.cpp:71-82 */
        for (int C = 0; C < m->natoms; ++C)
          if (C != A)
            s += -(double)core_charge(m->Z[C]) *
                 eri(m, blocks, A, ao[i].ang, A, ao[j].ang, C, 0, C, 0);
        h = s;
        if (i == j) h += ao[i].ang == 0 ? ELEM[zA].uss : ELEM[zA].upp; /* :84-92 */
      } else {                                                          /* :38-69 */
        double S = sto_overlap(zA, ao[i].ang, m->pos + 3 * A, zB, ao[j].ang, m->pos + 3 * B);
        double ba = ao[i].ang ? ELEM[zA].beta_p : ELEM[zA].beta_s;
        double bb = ao[j].ang ? ELEM[zB].beta_p : ELEM[zB].beta_s;
        h = (ba + bb) * S * 0.5;
      }
      H[tri(i) + j] = h;
    }
}

static double pfull(const double *P, int i, int j) { return i >= j ? P[tri(i) + j] : P[tri(j) + i]; }

/* Fock matrix F = H + G(P).  literal != 0: the reference's own O(N^4) double loop over every
 * (lam,sig) with two integral lookups per term (twoelectronmatrix.cpp:14-35,
 * fockmatrix.cpp:20-26).  literal == 0: the same sum restricted to its non-zero terms (the
 * lookup is zero unless both bra and ket pairs are one-atom pairs). */
static void build_fock(const mol_t *m, const ao_t *ao, const double *blocks, const double *H,
                       const double *P, double *F, int literal) {
  int n = m->nao;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      int A = ao[i].atom, B = ao[j].atom;
      double g = 0.0;
      if (literal) {
        for (int k = 0; k < n; ++k)
          for (int l = 0; l < n; ++l) {
            double t = eri(m, blocks, A, ao[i].ang, B, ao[j].ang, ao[k].atom, ao[k].ang,
                           ao[l].atom, ao[l].ang);
            t -= 0.5 * eri(m, blocks, A, ao[i].ang, ao[k].atom, ao[k].ang, B, ao[j].ang,
                           ao[l].atom, ao[l].ang);
            g += t * pfull(P, k, l);
          }
      } else if (A == B) {
        for (int C = 0; C < m->natoms; ++C) {
          int f = m->first[C], nc = nao_of(m->Z[C]);
          for (int k = f; k < f + nc; ++k)
            for (int l = f; l < f + nc; ++l)
              g += pfull(P, k, l) * eri(m, blocks, A, ao[i].ang, A, ao[j].ang, C, ao[k].ang, C,
                                        ao[l].ang);
        }
        int f = m->first[A], na = nao_of(m->Z[A]);
        for (int k = f; k < f + na; ++k)
          for (int l = f; l < f + na; ++l)
            g -= 0.5 * pfull(P, k, l) *
                 eri(m, blocks, A, ao[i].ang, A, ao[k].ang, A, ao[j].ang, A, ao[l].ang);
      } else {
        int fa = m->first[A], na = nao_of(m->Z[A]), fb = m->first[B], nb = nao_of(m->Z[B]);
        for (int k = fa; k < fa + na; ++k)
          for (int l = fb; l < fb + nb; ++l)
            g -= 0.5 * pfull(P, k, l) *
                 eri(m, blocks, A, ao[i].ang, A, ao[k].ang, B, ao[j].ang, B, ao[l].ang);
      }
      F[tri(i) + j] = H[tri(i) + j] + g;
    }
}

/* E_el = 1/2 Σ_ij P_ij (H_ij + F_ij) over the full matrix (electronicenergy.cpp:12-36) */
static double el_energy(int n, const double *H, const double *F, const double *P) {
  double e = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) e += 2.0 * (H[tri(i) + j] + F[tri(i) + j]) * P[tri(i) + j];
  for (int i = 0; i < n; ++i) e -= (H[tri(i) + i] + F[tri(i) + i]) * P[tri(i) + i];
  return 0.5 * e;
}

/* Core-core repulsion (corecorerepulsion.cpp:12-65): atoms A<B, Z_A Z_B (sA sA|sB sB) f(R),
 * R in Angstrom as bohr*0.529177249; N-H / O-H use the R*exp(-alpha_X R) form. */
static double core_core(const mol_t *m, const double *blocks) {
  double e = 0.0;
  for (int A = 0; A < m->natoms; ++A)
    for (int B = A + 1; B < m->natoms; ++B) {
      int zA = m->Z[A], zB = m->Z[B];
      double t = (double)(core_charge(zA) * core_charge(zB));
      t *= eri(m, blocks, A, 0, A, 0, B, 0, B, 0);
      double r = dist(m->pos + 3 * A, m->pos + 3 * B) * BOHR2ANG;
      double f;
      if (zB == 1 && (zA == 7 || zA == 8))
        f = 1.0 + r * exp(-ELEM[zA].alpha * r) + exp(-ELEM[zB].alpha * r);
      else if (zA == 1 && (zB == 7 || zB == 8))
        f = 1.0 + r * exp(-ELEM[zB].alpha * r) + exp(-ELEM[zA].alpha * r);
      else
        f = 1.0 + exp(-ELEM[zA].alpha * r) + exp(-ELEM[zB].alpha * r);
      e += t * f;
    }
  return e;
}

/* ---------------------------------------------------------------------------------------- */
/* LAPACK from the OpenBLAS in the SciPy wheel, as the reference links dsyev_ */
extern void scipy_dsyev_(char *jobz, char *uplo, int *n, double *a, int *lda, double *w,
                         double *work, int *lwork, int *info);

/* GetEigenValVecOfFmatrix (scfcalculation.cpp:171-203): column-major lower copy of F, dsyev */
static int eigh(int n, const double *F, double *C, double *w) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) C[(long)j * n + i] = F[tri(i) + j];
  char jobz = 'V', uplo = 'L';
  int lwork = -1, info = 0;
  double q;
  scipy_dsyev_(&jobz, &uplo, &n, C, &n, w, &q, &lwork, &info);
  lwork = (int)q;
  double *work = (double *)malloc(sizeof(double) * (lwork > 1 ? lwork : 1));
  scipy_dsyev_(&jobz, &uplo, &n, C, &n, w, work, &lwork, &info);
  free(work);
  return info;
}

/* P_ij = 2 Σ_{k<nocc} C_ik C_jk, C column-major (densitymatrix.cpp:22-47) */
static void density(int n, int nocc, const double *C, double *P) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0.0;
      for (int k = 0; k < nocc; ++k) s += C[(long)k * n + i] * C[(long)k * n + j];
      P[tri(i) + j] = 2.0 * s;
    }
}

/* ========================================================================================= */
/* Exported entry points (ctypes) */

int oracle_nao(int natoms, const int *Z) {
  int n = 0;
  for (int a = 0; a < natoms; ++a) {
    if (!supported(Z[a])) return -2;
    n += nao_of(Z[a]);
  }
  return n;
}

int oracle_nocc(int natoms, const int *Z) {
  int e = 0;
  for (int a = 0; a < natoms; ++a) e += core_charge(Z[a]);
  return e / 2;
}

long oracle_block_count(int natoms, const int *Z) {
  long off = 0;
  for (int a = 0; a < natoms; ++a)
    for (int b = 0; b <= a; ++b) off += block_rows(Z[a], Z[b]) * block_cols(Z[a], Z[b]);
  return off;
}

int oracle_integrals(int natoms, const int *Z, const double *xyz, double *blocks) {
  mol_t m;
  int rc = mol_init(&m, natoms, Z, xyz);
  if (rc) return rc;
  fill_blocks(&m, blocks);
  mol_free(&m);
  return 0;
}

int oracle_hcore(int natoms, const int *Z, const double *xyz, const double *blocks, double *H) {
  mol_t m;
  int rc = mol_init(&m, natoms, Z, xyz);
  if (rc) return rc;
  ao_t *ao = ao_table(&m);
  build_hcore(&m, ao, blocks, H);
  free(ao);
  mol_free(&m);
  return 0;
}

int oracle_overlap(int natoms, const int *Z, const double *xyz, double *S) {
  mol_t m;
  int rc = mol_init(&m, natoms, Z, xyz);
  if (rc) return rc;
  ao_t *ao = ao_table(&m);
  for (int i = 0; i < m.nao; ++i)
    for (int j = 0; j <= i; ++j) {
      int A = ao[i].atom, B = ao[j].atom;
      S[tri(i) + j] = sto_overlap(m.Z[A], ao[i].ang, m.pos + 3 * A, m.Z[B], ao[j].ang,
                                  m.pos + 3 * B);
    }
  free(ao);
  mol_free(&m);
  return 0;
}

int oracle_fock(int natoms, const int *Z, const double *blocks, const double *H, const double *P,
                double *F, int literal) {
  mol_t m;
  double *xyz = (double *)calloc(3 * (size_t)(natoms > 0 ? natoms : 1), sizeof(double));
  int rc = mol_init(&m, natoms, Z, xyz);
  free(xyz);
  if (rc) return rc;
  ao_t *ao = ao_table(&m);
  build_fock(&m, ao, blocks, H, P, F, literal);
  free(ao);
  mol_free(&m);
  return 0;
}

double oracle_energy(int nao, const double *H, const double *F, const double *P) {
  return el_energy(nao, H, F, P);
}

double oracle_core_core(int natoms, const int *Z, const double *xyz, const double *blocks) {
  mol_t m;
  if (mol_init(&m, natoms, Z, xyz)) return NAN;
  double e = core_core(&m, blocks);
  mol_free(&m);
  return e;
}

int oracle_density(int nao, int nocc, const double *C, double *P) {
  density(nao, nocc, C, P);
  return 0;
}

/* Full SCF as SCFCalculation::ComputeSCF (scfcalculation.cpp:66-165) with the threshold and
 * the step cap as arguments.  energies[] receives E_0..E_n_iter (max_iter+1 slots).  Any of
 * the output matrices may be NULL.  Returns 0, or the LAPACK info, or <0 on bad input. */
int oracle_scf(int natoms, const int *Z, const double *xyz, double tol, int max_iter,
               double *energies, int *n_iter, int *converged, double *e_el, double *e_cc,
               double *H_out, double *F_out, double *P_out, double *eig_out, int literal_fock) {
  mol_t m;
  int rc = mol_init(&m, natoms, Z, xyz);
  if (rc) return rc;
  int n = m.nao, nocc = oracle_nocc(natoms, Z);
  long np = tri(n);
  ao_t *ao = ao_table(&m);
  double *blocks = (double *)malloc(sizeof(double) * m.blk_total);
  double *H = (double *)malloc(sizeof(double) * np), *F = (double *)malloc(sizeof(double) * np);
  double *P = (double *)calloc(np, sizeof(double));
  double *C = (double *)malloc(sizeof(double) * (size_t)n * n);
  double *w = (double *)malloc(sizeof(double) * n);
  fill_blocks(&m, blocks);
  build_hcore(&m, ao, blocks, H);
  for (int i = 0; i < n; ++i) /* InitialGuess, densitymatrix.cpp:26-37 */
    P[tri(i) + i] = (double)core_charge(m.Z[ao[i].atom]) / nao_of(m.Z[ao[i].atom]);
  build_fock(&m, ao, blocks, H, P, F, literal_fock);
  double E = el_energy(n, H, F, P);
  energies[0] = E;
  int steps = 0, conv = 0, info = 0;
  for (int i = 0; i < n; ++i) w[i] = 0.0;
  while (!conv && steps < max_iter) {
    info = eigh(n, F, C, w);
    if (info) break;
    density(n, nocc, C, P);
    build_fock(&m, ao, blocks, H, P, F, literal_fock);
    double old = E;
    E = el_energy(n, H, F, P);
    energies[++steps] = E;
    conv = fabs(old - E) < tol; /* sameReal, mymath.h:70-75 */
  }
  *n_iter = steps;
  *converged = conv;
  *e_el = E;
  *e_cc = core_core(&m, blocks);
  if (H_out) memcpy(H_out, H, sizeof(double) * np);
  if (F_out) memcpy(F_out, F, sizeof(double) * np);
  if (P_out) memcpy(P_out, P, sizeof(double) * np);
  if (eig_out) memcpy(eig_out, w, sizeof(double) * n);
  free(blocks); free(H); free(F); free(P); free(C); free(w); free(ao);
  mol_free(&m);
  return info;
}
