// Test infrastructure only: a dump driver around the UNMODIFIED reference classes.
//
// It runs the reference's own stages in the order of src/App/semiGPU.cc:29-92 (reader, AO list,
// Alloc4AllTwoCenterIntegral, ComputeAllTwoCenterIntegral, Hcore, SCFCalculation,
// CoreCoreRepulsion) and the SCF loop of SCFCalculation::ComputeSCF
// (src/common/scfcalculation.cpp:66-146) step for step, calling the reference's own
// InitialGuess / GetEigenValVecOfFmatrix / DensityMatrix::ComputeMatrix /
// FockMatrix::ComputeMatrix / ElectronicEnergy::ComputeEnergy.  The only change is that the
// energy threshold (hard-coded 5e-3 eV at scfcalculation.cpp:77) and the step cap (100, :74)
// are arguments, so the oracle can be run at the 1e-6 eV tolerance of the workloads.
//
// Output: one JSON object with every intermediate printed at %.17g.
//   ref_driver geometry.xyz [--tol T] [--max-iter M] [--no-matrices] [--fock-only]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#define private public
#define protected public
#include "atom.h"
#include "atomicOrbitals.h"
#include "corecorerepulsion.h"
#include "electronicenergy.h"
#include "hcore.h"
#include "MNDO_parameters.h"
#include "mymath.h"
#include "mymemory.h"
#include "readxyzfile.h"
#include "scfcalculation.h"
#include "twocenterintegral.h"
#undef private
#undef protected

using Clock = std::chrono::high_resolution_clock;

static double secs(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

static void print_array(const char *key, const double *v, size_t n, bool last = false) {
  printf("\"%s\": [", key);
  for (size_t i = 0; i < n; ++i) printf(i ? ", %.17g" : "%.17g", v[i]);
  printf("]%s\n", last ? "" : ",");
}

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: ref_driver geometry.xyz [--tol T] [--max-iter M] [--no-matrices]\n");
    return 2;
  }
  std::string path = argv[1];
  double tol = 5.0e-3;
  unsigned max_iter = 100;
  bool matrices = true;
  for (int a = 2; a < argc; ++a) {
    if (!strcmp(argv[a], "--tol") && a + 1 < argc) tol = atof(argv[++a]);
    else if (!strcmp(argv[a], "--max-iter") && a + 1 < argc) max_iter = (unsigned)atoi(argv[++a]);
    else if (!strcmp(argv[a], "--no-matrices")) matrices = false;
  }

  ReadXYZFile reader;
  std::vector<Atom> molecule;
  if (!reader.GetValuesFromFile(path, molecule)) {
    printf("{\"error\": \"read\"}\n");
    return 1;
  }
  auto t0 = Clock::now();
  ListAtomicOrbitals infoAOs;
  infoAOs.SetOrbitals(molecule);
  const size_t nAOs = infoAOs.size();
  double ****ints = NULL;
  TwoCenterIntegral::Alloc4AllTwoCenterIntegral(molecule, ints);
  MNDOparameter parameters;
  TwoCenterIntegral twoCenInt(parameters);
  twoCenInt.ComputeAllTwoCenterIntegral(infoAOs, ints);
  auto t1 = Clock::now();
  Hcore hcore(parameters, infoAOs, ints);
  hcore.Alloc4Matrix("hcoreMatrix");
  hcore.ComputeMatrix();
  auto t2 = Clock::now();

  SCFCalculation scf(infoAOs, ints, hcore);
  scf.AllocSCFData();
  const size_t npk = nAOs * (nAOs + 1) / 2;

  // scfcalculation.cpp:67-70
  scf.InitialGuess();
  std::vector<double> P0(scf.Pmatrix->matrixHold_, scf.Pmatrix->matrixHold_ + npk);
  std::vector<double> F0(scf.Fmatrix->matrixHold_, scf.Fmatrix->matrixHold_ + npk);
  double E = ElectronicEnergy::ComputeEnergy(nAOs, hcore, *scf.Fmatrix, *scf.Pmatrix);
  std::vector<double> energies(1, E);
  bool converged = false;
  unsigned steps = 0;
  int lapack = 0;
  double t_fock = 0.0, t_eig = 0.0;
  auto t3 = Clock::now();
  // scfcalculation.cpp:82-141 with the threshold and the cap as arguments
  while (!converged && max_iter > steps) {
    auto a = Clock::now();
    lapack = scf.GetEigenValVecOfFmatrix();
    auto b = Clock::now();
    t_eig += secs(a, b);
    if (lapack != 0) break;
    scf.Pmatrix->ComputeMatrix();
    auto c = Clock::now();
    scf.Fmatrix->ComputeMatrix();
    auto d = Clock::now();
    t_fock += secs(c, d);
    double old = E;
    E = ElectronicEnergy::ComputeEnergy(nAOs, hcore, *scf.Fmatrix, *scf.Pmatrix);
    energies.push_back(E);
    converged = sameReal(old, E, tol);
    ++steps;
  }
  auto t4 = Clock::now();
  double Ecc = CoreCoreRepulsion::ComputeRepulsion(parameters, infoAOs, ints);
  auto t5 = Clock::now();

  int nelec = 0;
  for (size_t i = 0; i < molecule.size(); ++i) {
    int z = molecule[i].atomNumber;
    nelec += (z < 2) ? z : (z < 11 ? z - 2 : z - 10);
  }

  printf("{\n");
  printf("\"natoms\": %zu,\n\"nao\": %zu,\n\"nocc\": %d,\n", molecule.size(), nAOs, nelec / 2);
  printf("\"tol\": %.17g,\n\"max_iter\": %u,\n", tol, max_iter);
  printf("\"Z\": [");
  for (size_t i = 0; i < molecule.size(); ++i) printf(i ? ", %d" : "%d", molecule[i].atomNumber);
  printf("],\n\"xyz\": [");
  for (size_t i = 0; i < molecule.size(); ++i)
    for (int k = 0; k < 3; ++k)
      printf((i || k) ? ", %.17g" : "%.17g", molecule[i].atomCoordinates[k]);
  printf("],\n");
  if (matrices) {
    // Ragged integral storage in its own order: [A][B<=A], 1x1 / 1x10 / 10x10 row-major
    // (twocenterintegral.cpp:55-107).
    std::vector<double> blocks;
    for (size_t A = 0; A < molecule.size(); ++A)
      for (size_t B = 0; B <= A; ++B) {
        int za = molecule[A].atomNumber, zb = molecule[B].atomNumber;
        int r = (za > 1 && zb > 1) ? 10 : 1;
        int c = (za == 1 && zb == 1) ? 1 : 10;
        for (int i = 0; i < r; ++i)
          for (int j = 0; j < c; ++j) blocks.push_back(ints[A][B][i][j]);
      }
    print_array("blocks", blocks.data(), blocks.size());
    print_array("H", hcore.matrixHold_, npk);
    print_array("P0", P0.data(), npk);
    print_array("F0", F0.data(), npk);
    print_array("P", scf.Pmatrix->matrixHold_, npk);
    print_array("F", scf.Fmatrix->matrixHold_, npk);
    print_array("eig", scf.eigenVal, nAOs);
  }
  print_array("energies", energies.data(), energies.size());
  printf("\"lapack_info\": %d,\n", lapack);
  printf("\"n_iter\": %u,\n\"converged\": %s,\n", steps, converged ? "true" : "false");
  printf("\"E_el\": %.17g,\n\"E_cc\": %.17g,\n\"E_tot\": %.17g,\n", E, Ecc, E + Ecc);
  printf("\"t_integrals_s\": %.6g,\n\"t_hcore_s\": %.6g,\n\"t_scf_s\": %.6g,\n", secs(t0, t1),
         secs(t1, t2), secs(t3, t4));
  printf("\"t_fock_s\": %.6g,\n\"t_eig_s\": %.6g,\n\"t_corecore_s\": %.6g,\n", t_fock, t_eig,
         secs(t4, t5));
  printf("\"t_total_s\": %.6g\n}\n", secs(t0, t5));
  return 0;
}
