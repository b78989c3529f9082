// semiGPU geometry.xyz — the reference CLI (src/App/semiGPU.cc:20-116) on the B200 engine: the
// same stages in the same order and the same printout.  The input file is the last argument,
// as in the reference; optional flags before it:
//   --tol T       SCF energy threshold in eV (default 5e-3, the reference's hard-coded value)
//   --max-iter M  SCF step cap (default 100)
//   --heat        also print the heat of formation (not printed by the reference)
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <vector>

#include "semigpu.h"
#include "semigpu_b200.h"

using std::cout;
using std::endl;
using std::setw;

int main(int argc, char* argv[]) {
  auto start = std::chrono::high_resolution_clock::now();
  if (argc < 2) {
    cout << "usage: semiGPU [--tol T] [--max-iter M] geometry.xyz" << endl;
    return EXIT_FAILURE;
  }
  double tol = 5.0e-3;
  unsigned max_iter = 100;
  bool heat = false;
  for (int a = 1; a + 1 < argc; ++a) {
    if (!strcmp(argv[a], "--tol")) tol = atof(argv[++a]);
    else if (!strcmp(argv[a], "--max-iter")) max_iter = (unsigned)atoi(argv[++a]);
    else if (!strcmp(argv[a], "--heat")) heat = true;
  }
  string filename_molecule = argv[argc - 1];
  cout << "XYZ file : " << filename_molecule << endl;

  ReadXYZFile reader;
  vector<Atom> molecule;
  if (!(reader.GetValuesFromFile(filename_molecule, molecule))) {
    cout << "Problem to read xyz file " << endl;
    return EXIT_FAILURE;
  } else {
    cout << "Read XYZ file successful" << endl;
  }
  Atom::PrintGeometry(molecule);
  ScreenUtils::PrintScrStarLine();

  ListAtomicOrbitals infoAOs;
  infoAOs.SetOrbitals(molecule);
  double**** all2CenterIntegrals = NULL;
  if (!(TwoCenterIntegral::Alloc4AllTwoCenterIntegral(molecule, all2CenterIntegrals))) {
    cout << "Problem to alloc all2CenterIntegrals" << endl;
    return EXIT_FAILURE;
  } else {
    cout << "Correct Alloc: all2CenterIntegrals" << endl;
  }
  MNDOparameter parameters;
  TwoCenterIntegral twoCenInt(parameters);
  twoCenInt.ComputeAllTwoCenterIntegral(infoAOs, all2CenterIntegrals);
  TwoCenterIntegral::To_device(molecule, all2CenterIntegrals);
  if (semigpu::last_status() != 0) {
    cout << "Problem computing all2CenterIntegrals: " << semigpu::last_error() << endl;
    return EXIT_FAILURE;
  }

  Hcore hcore(parameters, infoAOs, all2CenterIntegrals);
  if (hcore.Alloc4Matrix("hcoreMatrix")) {
    cout << "Correct Alloc: hcoreMatrix" << endl;
  } else {
    cout << "Bad Alloc: hcoreMatrix " << endl;
  }
  hcore.ComputeMatrix();
  SCFCalculation SCFprocess(infoAOs, all2CenterIntegrals, hcore);
  SCFprocess.thresholdEnergy = tol;
  SCFprocess.maxSCFSteps = max_iter;
  if (SCFprocess.AllocSCFData()) {
    cout << "Correct Alloc: SCFData" << endl;
  } else {
    cout << "Bad Alloc: SCFData " << endl;
    return EXIT_FAILURE;
  }
  ScreenUtils::PrintScrStarLine();
  SCFprocess.ComputeSCF();
  if (semigpu::last_status() < 0) {
    cout << "SCF failed: " << semigpu::last_error() << endl;
    return EXIT_FAILURE;
  }

  double electronicEnergy = SCFprocess.finalEnergy;
  ScreenUtils::PrintScrStarLine();
  cout << "  Electronic Energy = " << setw(10) << electronicEnergy << " eV" << endl;
  ScreenUtils::PrintScrStarLine();
  double coreCoreRepulsionEnergy =
      CoreCoreRepulsion::ComputeRepulsion(parameters, infoAOs, all2CenterIntegrals);
  cout << "Core-Core Repulsion = " << setw(10) << coreCoreRepulsionEnergy << " eV" << endl;
  ScreenUtils::PrintScrStarLine();
  cout << "       Total Energy = " << setw(10) << electronicEnergy + coreCoreRepulsionEnergy
       << " eV" << endl;
  ScreenUtils::PrintScrStarLine();
  if (heat) {
    double dhf = 0.0;
    sgb_heat_of_formation((int)infoAOs.Z.size(), infoAOs.Z.data(),
                          electronicEnergy + coreCoreRepulsionEnergy, &dhf);
    cout << "  Heat of Formation = " << setw(10) << dhf << " kcal/mol" << endl;
    ScreenUtils::PrintScrStarLine();
  }

  cout << "Dealloc array: SCFData" << endl;
  SCFprocess.DeallocSCFData();
  cout << "Dealloc array: hcoreMatrix" << endl;
  hcore.Dealloc4Matrix();
  cout << "Dealloc array: all2CenterIntegral" << endl;
  TwoCenterIntegral::Dealloc4AllTwoCenterIntegral(molecule, all2CenterIntegrals);

  auto end = std::chrono::high_resolution_clock::now();
  auto duration = std::chrono::duration_cast<std::chrono::milliseconds>(end - start);
  ScreenUtils::PrintScrStarLine();
  double duration_sec = static_cast<double>(duration.count()) / 1000.0;
  cout << "Time taken for calculation: " << duration_sec << " s" << endl;
  return EXIT_SUCCESS;
}
