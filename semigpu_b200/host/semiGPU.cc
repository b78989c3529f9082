// semiGPU geometry.xyz — the reference CLI (src/App/semiGPU.cc:20-116) on the B200 engine: the
// same stages in the same order and the same printout.  The input file is the last argument,
// as in the reference; optional flags before it:
//   --tol T       SCF energy threshold in eV (default 5e-3, the reference's hard-coded value)
//   --max-iter M  SCF step cap (default 100)
//   --heat        also print the heat of formation (not printed by the reference)
//   --frames      the file holds several XYZ frames (an ensemble or a trajectory): all of them
//                 run as one batched launch, one result line per frame (not in the reference)
//   --json        with --frames, one JSON object per frame instead of the text line
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

namespace {

// JSON string body: quotes, backslashes and control characters escaped.
std::string json_escape(const std::string& s) {
  std::string o;
  for (char ch : s) {
    const unsigned char c = (unsigned char)ch;
    if (c == '"' || c == '\\') {
      o += '\\';
      o += ch;
    } else if (c < 0x20) {
      char buf[8];
      snprintf(buf, sizeof buf, "\\u%04x", c);
      o += buf;
    } else {
      o += ch;
    }
  }
  return o;
}

// --frames: every frame of the file through sgb_run_molecules (one batch), a line per frame.
int run_frames(const string& file, double tol, unsigned max_iter, bool heat, bool json) {
  ReadXYZFile reader;
  vector<vector<Atom>> frames;
  vector<string> comments;
  if (!reader.GetFramesFromFile(file, frames, comments)) {
    cout << "Problem to read xyz file " << endl;
    return EXIT_FAILURE;
  }
  sgb_ctx* ctx = semigpu::context();
  if (!ctx) {
    cout << "No device context: " << semigpu::last_error() << endl;
    return EXIT_FAILURE;
  }
  const int nf = (int)frames.size();
  vector<int> natoms(nf), Z;
  vector<double> xyz;
  for (int f = 0; f < nf; ++f) {
    natoms[f] = (int)frames[f].size();
    for (Atom& a : frames[f]) {
      Z.push_back(a.atomNumber);
      xyz.push_back(a.getXCoordinate());
      xyz.push_back(a.getYCoordinate());
      xyz.push_back(a.getZCoordinate());
    }
  }
  vector<double> eel(nf), ecc(nf);
  vector<int> it(nf), cv(nf), st(nf);
  const int rc = sgb_run_molecules(ctx, nf, natoms.data(), Z.data(), xyz.data(), tol,
                                   (int)max_iter, eel.data(), ecc.data(), it.data(), cv.data(),
                                   st.data());
  if (rc != SGB_OK) {
    cout << "Batch failed: " << sgb_status_string(rc) << ": " << sgb_last_error(ctx) << endl;
    return EXIT_FAILURE;
  }
  if (!json) {
    cout << "XYZ file : " << file << endl;
    cout << "Frames   : " << nf << endl;
    ScreenUtils::PrintScrStarLine();
  }
  const int* zf = Z.data();
  bool all_ok = true;
  for (int f = 0; f < nf; ++f) {
    const double et = eel[f] + ecc[f];
    double dhf = 0.0;
    if (heat && st[f] == SGB_OK) sgb_heat_of_formation(natoms[f], zf, et, &dhf);
    zf += natoms[f];
    all_ok = all_ok && st[f] == SGB_OK && cv[f];
    if (json) {
      cout << std::setprecision(12) << "{\"frame\": " << f << ", \"comment\": \""
           << json_escape(comments[f]) << "\", \"natoms\": " << natoms[f]
           << ", \"E_el\": " << eel[f] << ", \"E_cc\": " << ecc[f] << ", \"E_tot\": " << et
           << ", \"n_iter\": " << it[f] << ", \"converged\": " << (cv[f] ? "true" : "false")
           << ", \"status\": " << st[f];
      if (heat) cout << ", \"heat_of_formation_kcal_mol\": " << dhf;
      cout << "}" << endl;
    } else {
      cout << "frame " << setw(5) << f << "  atoms " << setw(5) << natoms[f] << "  E_el "
           << setw(16) << std::setprecision(10) << eel[f] << "  E_cc " << setw(16) << ecc[f]
           << "  E_tot " << setw(16) << et << " eV  steps " << setw(3) << it[f]
           << (cv[f] ? "  converged" : "  NOT converged");
      if (heat) cout << "  dHf " << dhf << " kcal/mol";
      if (st[f] != SGB_OK) cout << "  status " << sgb_status_string(st[f]);
      cout << endl;
    }
  }
  return all_ok ? EXIT_SUCCESS : EXIT_FAILURE;
}

}  // namespace

int main(int argc, char* argv[]) {
  auto start = std::chrono::high_resolution_clock::now();
  if (argc < 2) {
    cout << "usage: semiGPU [--tol T] [--max-iter M] [--heat] [--frames [--json]] geometry.xyz"
         << endl;
    return EXIT_FAILURE;
  }
  double tol = 5.0e-3;
  unsigned max_iter = 100;
  bool heat = false, frames = false, json = false;
  for (int a = 1; a + 1 < argc; ++a) {
    if (!strcmp(argv[a], "--tol")) tol = atof(argv[++a]);
    else if (!strcmp(argv[a], "--max-iter")) max_iter = (unsigned)atoi(argv[++a]);
    else if (!strcmp(argv[a], "--heat")) heat = true;
    else if (!strcmp(argv[a], "--frames")) frames = true;
    else if (!strcmp(argv[a], "--json")) json = true;
  }
  string filename_molecule = argv[argc - 1];
  if (frames) return run_frames(filename_molecule, tol, max_iter, heat, json);
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
