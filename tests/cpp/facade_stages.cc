// Test program for the C++ host API (semigpu_b200/host/semigpu.h): the reference's stage
// sequence (src/App/semiGPU.cc:29-92), then two checks a user of the reference classes relies
// on -- ElectronicEnergy::ComputeEnergy on the SCF's final matrices (electronicenergy.cpp:12-36)
// and the host mirror of the integrals through TwoCenterIntegral::GetValueFromArray, used in
// the reference's literal Fock sum F_uv = H_uv + sum_ls P_ls [(uv|ls) - 1/2 (ul|vs)]
// (twoelectronmatrix.cpp:14-35) and compared with the device Fock matrix.
// Prints one JSON line last.
//   facade_stages geometry.xyz [tol]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "semigpu.h"

static size_t packed(size_t i, size_t j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  ReadXYZFile reader;
  vector<Atom> molecule;
  if (!reader.GetValuesFromFile(argv[1], molecule)) return 3;
  ListAtomicOrbitals infoAOs;
  infoAOs.SetOrbitals(molecule);
  const size_t n = infoAOs.size();
  double**** ints = nullptr;
  if (!TwoCenterIntegral::Alloc4AllTwoCenterIntegral(molecule, ints)) return 4;
  MNDOparameter parameters;
  TwoCenterIntegral twoCenInt(parameters);
  twoCenInt.ComputeAllTwoCenterIntegral(infoAOs, ints);
  Hcore hcore(parameters, infoAOs, ints);
  hcore.Alloc4Matrix("hcoreMatrix");
  hcore.ComputeMatrix();
  SCFCalculation scf(infoAOs, ints, hcore);
  scf.thresholdEnergy = argc > 2 ? atof(argv[2]) : 5.0e-3;
  if (!scf.AllocSCFData()) return 5;
  scf.ComputeSCF();
  const double e_facade =
      ElectronicEnergy::ComputeEnergy(n, hcore, *scf.Fmatrix, *scf.Pmatrix);
  const double* H = hcore.matrixHold_;
  const double* P = scf.Pmatrix->matrixHold_;
  const double* F = scf.Fmatrix->matrixHold_;
  double max_df = 0.0;
  for (size_t u = 0; u < n; ++u)
    for (size_t v = 0; v <= u; ++v) {
      double g = 0.0;
      for (size_t l = 0; l < n; ++l)
        for (size_t s = 0; s < n; ++s) {
          const AtomicOrbital &U = infoAOs.orbital[u], &V = infoAOs.orbital[v],
                              &L = infoAOs.orbital[l], &S = infoAOs.orbital[s];
          g += P[packed(l, s)] * (TwoCenterIntegral::GetValueFromArray(U, V, L, S, ints) -
                                  0.5 * TwoCenterIntegral::GetValueFromArray(U, L, V, S, ints));
        }
      max_df = std::fmax(max_df, std::fabs(H[packed(u, v)] + g - F[packed(u, v)]));
    }
  const double ecc = CoreCoreRepulsion::ComputeRepulsion(parameters, infoAOs, ints);
  printf("{\"nao\": %zu, \"steps\": %u, \"converged\": %d, \"final_energy\": %.17g, "
         "\"energy_recomputed\": %.17g, \"e_cc\": %.17g, \"max_abs_dF_lookup\": %.17g}\n",
         n, scf.SCFSteps, scf.energyConverge ? 1 : 0, scf.finalEnergy, e_facade, ecc, max_df);
  scf.DeallocSCFData();
  hcore.Dealloc4Matrix();
  TwoCenterIntegral::Dealloc4AllTwoCenterIntegral(molecule, ints);
  return 0;
}
