// Host façade implementation: reference class names over the engine's C ABI.
#include "semigpu.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>

#include "semigpu_b200.h"

using std::cout;
using std::endl;
using std::setw;

namespace {

sgb_ctx* g_ctx = nullptr;
int g_status = 0;
std::string g_error;

bool check(int rc, const char* what) {
  if (rc == SGB_OK) return true;
  g_status = rc;
  g_error = std::string(what) + ": " + sgb_status_string(rc) + " (" +
            (g_ctx ? sgb_last_error(g_ctx) : "no context") + ")";
  std::cerr << "semigpu: " << g_error << std::endl;
  return false;
}

// Element symbols Z = 1..109 (the reference reader accepts any of them and marks the rest
// invalid, atom.cpp:77-88; the engine itself only has MNDO parameters for H, C, N, O).
const char* const kSymbols[] = {
    "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",  "S",
    "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge",
    "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd",
    "In", "Sn", "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd",
    "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au", "Hg",
    "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U",  "Np", "Pu", "Am", "Cm",
    "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr", "Rf", "Db", "Sg", "Bh", "Hs", "Mt"};
constexpr int kNumSymbols = 109;

int core_charge(int z) { return z < 2 ? z : (z < 11 ? z - 2 : (z < 19 ? z - 10 : -1)); }

}  // namespace

namespace semigpu {
sgb_ctx* context() {
  if (!g_ctx) {
    const char* dev = getenv("SEMIGPU_DEVICE");
    if (!check(sgb_ctx_create(dev ? atoi(dev) : 0, 0, &g_ctx), "sgb_ctx_create")) g_ctx = nullptr;
  }
  return g_ctx;
}
int last_status() { return g_status; }
const char* last_error() { return g_error.c_str(); }
}  // namespace semigpu

// ---- Atom ---------------------------------------------------------------------------------
Atom::Atom()
    : atomNumber(0), atomCoordinates{0, 0, 0}, atomWeight(0), atomValenceElectrons(0),
      statusData(true) {}
void Atom::setCoordinates(double x, double y, double z) {
  atomCoordinates[0] = x; atomCoordinates[1] = y; atomCoordinates[2] = z;
}
void Atom::setCoordinates(vector<double> v) { setCoordinates(v[0], v[1], v[2]); }
void Atom::setCoordinates(double (&v)[3]) { setCoordinates(v[0], v[1], v[2]); }
double Atom::getXCoordinate() { return atomCoordinates[0]; }
double Atom::getYCoordinate() { return atomCoordinates[1]; }
double Atom::getZCoordinate() { return atomCoordinates[2]; }
void Atom::setAtomSymbol(string s) {
  atomNumber = 0;
  for (int i = 0; i < kNumSymbols; ++i)
    if (s == kSymbols[i]) { atomNumber = i + 1; break; }
  atomSymbol = s;
  if (atomNumber == 0) {
    atomSymbol += " Invalid atomic symbol";
    statusData = false;
  }
}
void Atom::setAtomNumber(int z) {
  if (z > 0 && z <= kNumSymbols) {
    atomNumber = z;
    atomSymbol = kSymbols[z - 1];
  } else {
    atomNumber = 0;
    atomSymbol = " Invalid atomic number";
    statusData = false;
  }
}
void Atom::PrintGeometry(const vector<Atom>& molecule) {
  cout << "Geometry :" << endl;
  for (const Atom& a : molecule) {
    cout << setw(3) << a.atomSymbol;
    cout << setw(10) << a.atomCoordinates[0];
    cout << setw(10) << a.atomCoordinates[1];
    cout << setw(10) << a.atomCoordinates[2] << endl;
  }
}

// ---- ReadXYZFile (readxyzfile.cpp:27-133: count, comment line, symbol-or-number rows) ----
ReadXYZFile::ReadXYZFile() : Natoms(0), open_without_problems(true) {}

bool ReadXYZFile::GetFramesFromFile(string filename, vector<vector<Atom>>& frames,
                                    vector<string>& comments) {
  frames.clear();
  comments.clear();
  std::ifstream f(filename.c_str());
  if (!f.good()) {
    cout << "Error: File " << filename << " could not be opened...\n";
    open_without_problems = false;
    return false;
  }
  open_without_problems = false;
  std::string line;
  while (std::getline(f, line)) {
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;  // between frames
    std::stringstream head(line);
    int n = 0;
    if (!(head >> n) || n <= 0) {
      cout << "Error: frame " << frames.size() << " of " << filename
           << " does not start with an atom count" << endl;
      return false;
    }
    std::string comment;
    std::getline(f, comment);
    vector<Atom> mol(n, Atom());
    for (int i = 0; i < n; ++i) {
      if (!std::getline(f, line)) {
        cout << "Error: frame " << frames.size() << " of " << filename << " ends after " << i
             << " of " << n << " atoms" << endl;
        return false;
      }
      std::stringstream ls(line);
      std::string tok;
      double x = 0, y = 0, z = 0;
      if (!(ls >> tok >> x >> y >> z)) {
        cout << "Error: frame " << frames.size() << " of " << filename << ", atom " << i
             << ": expected 'element x y z'" << endl;
        return false;
      }
      if (tok.find_first_not_of("0123456789") == std::string::npos)
        mol[i].setAtomNumber(atoi(tok.c_str()));
      else
        mol[i].setAtomSymbol(tok);
      mol[i].setCoordinates(x, y, z);
      if (!mol[i].statusData) {
        cout << "Error: frame " << frames.size() << " of " << filename << ", atom " << i
             << ": unknown element " << tok << endl;
        return false;
      }
    }
    if (!comment.empty() && comment.back() == '\r') comment.pop_back();
    frames.push_back(std::move(mol));
    comments.push_back(comment);
  }
  Natoms = frames.empty() ? 0 : (int)frames.back().size();
  open_without_problems = !frames.empty();
  return open_without_problems;
}

bool ReadXYZFile::GetValuesFromFile(string filename, vector<Atom>& molecule) {
  std::ifstream f(filename.c_str());
  if (!f.good()) {
    cout << "Error: File " << filename << " could not be opened...\n";
    open_without_problems = false;
    return false;
  }
  std::string line;
  Natoms = 0;
  f >> Natoms;
  if (Natoms <= 0) {
    cout << "Error: File " << filename << " does not have the XYZ format..." << endl;
    open_without_problems = false;
    return false;
  }
  std::getline(f, line);  // rest of the count line
  std::getline(f, line);  // comment
  std::stringstream rest;
  rest << f.rdbuf();
  std::string tok;
  molecule.assign(Natoms, Atom());
  bool numeric = false;
  {
    std::streampos p = rest.tellg();
    int probe;
    numeric = static_cast<bool>(rest >> probe);
    rest.clear();
    rest.seekg(p);
  }
  for (int i = 0; i < Natoms; ++i) {
    double x = 0, y = 0, z = 0;
    if (numeric) {
      int zn = 0;
      rest >> zn >> x >> y >> z;
      molecule[i].setAtomNumber(zn);
    } else {
      rest >> tok >> x >> y >> z;
      molecule[i].setAtomSymbol(tok);
    }
    molecule[i].setCoordinates(x, y, z);
  }
  open_without_problems = true;
  for (const Atom& a : molecule)
    if (!a.statusData) open_without_problems = false;
  return open_without_problems;
}

// ---- AO list (atomicOrbitals.cpp:76-119) --------------------------------------------------
AtomicOrbital::AtomicOrbital()
    : indexAtom(0), element(0), angularMomentum{0, 0, 0}, angularMomentumInt(0), indexAO(0),
      coordinates{0, 0, 0} {}
int AtomicOrbital::GetCoreCharge() const { return core_charge(element); }
int AtomicOrbital::GetAOsSize() const { return element < 2 ? 1 : (element < 11 ? 4 : -1); }

ListAtomicOrbitals::ListAtomicOrbitals()
    : orbital(nullptr), statusData(true), totalOrbitals_(0), mol_(nullptr) {}
ListAtomicOrbitals::~ListAtomicOrbitals() {
  if (mol_) sgb_mol_destroy(mol_);
  delete[] orbital;
}
size_t ListAtomicOrbitals::size() const { return totalOrbitals_; }

void ListAtomicOrbitals::SetOrbitals(const vector<Atom>& molecule) {
  Z.clear();
  xyz.clear();
  size_t total = 0;
  for (const Atom& a : molecule) {
    total += a.atomNumber <= 2 ? 1 : 4;
    if (a.atomNumber > 18) statusData = false;
    Z.push_back(a.atomNumber);
    for (int k = 0; k < 3; ++k) xyz.push_back(a.atomCoordinates[k]);
  }
  delete[] orbital;
  orbital = new AtomicOrbital[total];
  totalOrbitals_ = total;
  size_t k = 0;
  for (size_t i = 0; i < molecule.size(); ++i) {
    const int n = molecule[i].atomNumber <= 2 ? 1 : 4;
    for (int t = 0; t < n; ++t, ++k) {
      AtomicOrbital& o = orbital[k];
      o.indexAtom = (int)i;
      o.element = molecule[i].atomNumber;
      o.angularMomentumInt = t;
      for (int c = 0; c < 3; ++c) o.angularMomentum[c] = (t == c + 1);
      o.indexAO = (int)k;
      for (int c = 0; c < 3; ++c) o.coordinates[c] = molecule[i].atomCoordinates[c] * 1.8897259886;
    }
  }
  if (mol_) {
    sgb_mol_destroy(mol_);
    mol_ = nullptr;
  }
}

sgb_mol* ListAtomicOrbitals::device() const {
  if (!mol_ && semigpu::context()) {
    if (!check(sgb_mol_create(semigpu::context(), (int)Z.size(), Z.data(), xyz.data(), &mol_),
               "sgb_mol_create"))
      mol_ = nullptr;
  }
  return mol_;
}

// ---- MNDOparameter: the engine's tables, laid out as the reference's arrays indexed by Z ---
MNDOparameter::MNDOparameter() : countParameter_(20) {
  double** scalars[] = {&uss, &upp, &zs, &betaS, &betaP, &alpha, &gss, &gpp, &gsp, &gp2, &hsp,
                        &heat, &eisol};
  for (double** p : scalars) *p = new double[countParameter_]();
  dd = new double*[countParameter_];
  pp = new double*[countParameter_];
  for (unsigned i = 0; i < countParameter_; ++i) {
    dd[i] = new double[2]();
    pp[i] = new double[3]();
  }
  for (int z : {1, 6, 7, 8}) {
    double v[SGB_PARAM_COUNT];
    if (sgb_mndo_parameters(z, v) != SGB_OK) continue;
    uss[z] = v[SGB_P_USS]; upp[z] = v[SGB_P_UPP]; zs[z] = v[SGB_P_ZS];
    betaS[z] = v[SGB_P_BETAS]; betaP[z] = v[SGB_P_BETAP]; alpha[z] = v[SGB_P_ALPHA];
    gss[z] = v[SGB_P_GSS]; gpp[z] = v[SGB_P_GPP]; gsp[z] = v[SGB_P_GSP]; gp2[z] = v[SGB_P_GP2];
    hsp[z] = v[SGB_P_HSP]; dd[z][0] = v[SGB_P_DD1]; dd[z][1] = v[SGB_P_DD2];
    pp[z][0] = v[SGB_P_RHO0]; pp[z][1] = v[SGB_P_RHO1]; pp[z][2] = v[SGB_P_RHO2];
    heat[z] = v[SGB_P_HEAT]; eisol[z] = v[SGB_P_EISOL];
  }
}
MNDOparameter::~MNDOparameter() {
  for (double* p : {uss, upp, zs, betaS, betaP, alpha, gss, gpp, gsp, gp2, hsp, heat, eisol})
    delete[] p;
  for (unsigned i = 0; i < countParameter_; ++i) {
    delete[] dd[i];
    delete[] pp[i];
  }
  delete[] dd;
  delete[] pp;
}

// ---- TwoCenterIntegral ------------------------------------------------------------------------
TwoCenterIntegral::TwoCenterIntegral(MNDOparameter& p) : parameter(&p) {}

static int block_rows(int za, int zb) { return (za > 1 && zb > 1) ? 10 : 1; }
static int block_cols(int za, int zb) { return (za == 1 && zb == 1) ? 1 : 10; }

bool TwoCenterIntegral::Alloc4AllTwoCenterIntegral(const vector<Atom>& molecule, double****& ints) {
  const size_t n = molecule.size();
  ints = new double***[n];
  for (size_t A = 0; A < n; ++A) {
    ints[A] = new double**[A + 1];
    for (size_t B = 0; B <= A; ++B) {
      const int r = block_rows(molecule[A].atomNumber, molecule[B].atomNumber);
      const int c = block_cols(molecule[A].atomNumber, molecule[B].atomNumber);
      ints[A][B] = new double*[r];
      for (int i = 0; i < r; ++i) ints[A][B][i] = new double[c]();
    }
  }
  return true;
}

bool TwoCenterIntegral::Dealloc4AllTwoCenterIntegral(const vector<Atom>& molecule, double****& ints) {
  if (!ints) return false;
  const size_t n = molecule.size();
  for (size_t A = 0; A < n; ++A) {
    for (size_t B = 0; B <= A; ++B) {
      const int r = block_rows(molecule[A].atomNumber, molecule[B].atomNumber);
      for (int i = 0; i < r; ++i) delete[] ints[A][B][i];
      delete[] ints[A][B];
    }
    delete[] ints[A];
  }
  delete[] ints;
  ints = nullptr;
  return true;
}

void TwoCenterIntegral::ComputeAllTwoCenterIntegral(const ListAtomicOrbitals& infoAOs,
                                                    double****& ints) {
  sgb_mol* m = infoAOs.device();
  if (!m || !check(sgb_two_center(semigpu::context(), m), "sgb_two_center")) return;
  int natoms = 0, nao = 0, nocc = 0;
  long long nblk = 0;
  sgb_mol_info(m, &natoms, &nao, &nocc, &nblk);
  vector<double> flat((size_t)nblk);
  if (!check(sgb_get(semigpu::context(), m, SGB_BLOCKS, flat.data(), flat.size()), "sgb_get"))
    return;
  if (!ints) return;  // device-only use
  size_t off = 0;
  for (int A = 0; A < natoms; ++A)
    for (int B = 0; B <= A; ++B) {
      const int r = block_rows(infoAOs.Z[A], infoAOs.Z[B]), c = block_cols(infoAOs.Z[A], infoAOs.Z[B]);
      for (int i = 0; i < r; ++i)
        for (int j = 0; j < c; ++j) ints[A][B][i][j] = flat[off++];
    }
}

void TwoCenterIntegral::To_device(const vector<Atom>&, double****&) {
  // the integrals are computed on, and stay in, device memory
}

// Lookup of the mirrored blocks with the reference's semantics (twocenterintegral.cpp:285-386)
double TwoCenterIntegral::GetValueFromArray(const AtomicOrbital& a, const AtomicOrbital& b,
                                            const AtomicOrbital& c, const AtomicOrbital& d,
                                            double**** ints) {
  if (a.indexAtom != b.indexAtom || c.indexAtom != d.indexAtom) return 0.0;
  int A = a.indexAtom, C = c.indexAtom, ta = a.angularMomentumInt, tb = b.angularMomentumInt,
      tc = c.angularMomentumInt, td = d.angularMomentumInt, zA = a.element, zC = c.element;
  if (A < C) {
    std::swap(A, C); std::swap(ta, tc); std::swap(tb, td); std::swap(zA, zC);
  }
  auto pair = [](int x, int y) { if (x > y) std::swap(x, y); return y * (y + 1) / 2 + x; };
  if (zA > 1 && zC > 1) return ints[A][C][pair(ta, tb)][pair(tc, td)];
  if (zA == 1 && zC == 1) return ints[A][C][0][0];
  return ints[A][C][0][zA > 1 ? pair(ta, tb) : pair(tc, td)];
}

// ---- matrices ---------------------------------------------------------------------------------
BaseMatrix::BaseMatrix() : matrixSize_(0), matrixHold_(nullptr), array1DSize_(0) {}
BaseMatrix::BaseMatrix(size_t n) : matrixSize_(n), matrixHold_(nullptr), array1DSize_(n * (n + 1) / 2) {}
BaseMatrix::~BaseMatrix() {}
bool BaseMatrix::Alloc4Matrix(string) {
  delete[] matrixHold_;
  matrixHold_ = new double[array1DSize_]();
  return matrixHold_ != nullptr;
}
bool BaseMatrix::Dealloc4Matrix() {
  delete[] matrixHold_;
  matrixHold_ = nullptr;
  return true;
}
void BaseMatrix::ComputeMatrix() {}

Hcore::Hcore(const MNDOparameter&, const ListAtomicOrbitals& infoAOs, double****)
    : BaseMatrix(infoAOs.size()), infoAOs_(&infoAOs) {}

void Hcore::ComputeMatrix() {
  sgb_mol* m = infoAOs_->device();
  if (!m || !check(sgb_hcore(semigpu::context(), m), "sgb_hcore")) return;
  if (matrixHold_) check(sgb_get(semigpu::context(), m, SGB_HCORE, matrixHold_, array1DSize_), "sgb_get");
}

DensityMatrix::DensityMatrix(const ListAtomicOrbitals& infoAOs, const double*, const size_t nAOs)
    : BaseMatrix(nAOs), infoAOs_(&infoAOs), guessSwitch_(false) {}
void DensityMatrix::GuessDensityMatrixSwitch(bool g) { guessSwitch_ = g; }
void DensityMatrix::ComputeMatrix() {
  if (!matrixHold_) return;
  if (guessSwitch_) {
    for (size_t k = 0; k < array1DSize_; ++k) matrixHold_[k] = 0.0;
    for (size_t i = 0; i < matrixSize_; ++i) {
      const AtomicOrbital& o = infoAOs_->orbital[i];
      matrixHold_[i * (i + 1) / 2 + i] = (double)o.GetCoreCharge() / o.GetAOsSize();
    }
    return;
  }
  sgb_mol* m = infoAOs_->device();
  if (m) check(sgb_get(semigpu::context(), m, SGB_DENSITY, matrixHold_, array1DSize_), "sgb_get");
}

FockMatrix::FockMatrix(const ListAtomicOrbitals& infoAOs, const Hcore&, const DensityMatrix& P,
                       double****&)
    : BaseMatrix(infoAOs.size()), lastElectronicEnergy(0.0), infoAOs_(&infoAOs), Pmatrix_(&P) {}

void FockMatrix::ComputeMatrix() {
  sgb_mol* m = infoAOs_->device();
  if (!m || !matrixHold_ || !Pmatrix_->matrixHold_) return;
  check(sgb_fock(semigpu::context(), m, Pmatrix_->matrixHold_, matrixHold_, &lastElectronicEnergy),
        "sgb_fock");
}

// ---- ElectronicEnergy -------------------------------------------------------------------------
ElectronicEnergy::ElectronicEnergy() {}

double ElectronicEnergy::ComputeEnergy(const size_t& nAOs, const Hcore& hcore,
                                       const FockMatrix& Fmatrix, const DensityMatrix& Pmatrix) {
  if (!hcore.matrixHold_ || !Fmatrix.matrixHold_ || !Pmatrix.matrixHold_ || nAOs == 0) return 0.0;
  double e = 0.0;
  check(sgb_electronic_energy(semigpu::context(), (int)nAOs, hcore.matrixHold_,
                              Fmatrix.matrixHold_, Pmatrix.matrixHold_, &e),
        "sgb_electronic_energy");
  return e;
}

// ---- SCFCalculation ---------------------------------------------------------------------------
SCFCalculation::SCFCalculation(const ListAtomicOrbitals& infoAOs, double****& ints, const Hcore& h)
    : eigenVec(nullptr), eigenVal(nullptr), Pmatrix(nullptr), Fmatrix(nullptr), finalEnergy(0.0),
      energyConverge(false), thresholdEnergy(5.0e-3), maxSCFSteps(100), SCFSteps(0),
      infoAOs_(&infoAOs), nAOs_(infoAOs.size()), all2CIntegral_(ints), hcore_(&h) {}

bool SCFCalculation::AllocSCFData() {
  eigenVec = new double[nAOs_ * nAOs_]();
  eigenVal = new double[nAOs_]();
  Pmatrix = new DensityMatrix(*infoAOs_, eigenVec, nAOs_);
  Fmatrix = new FockMatrix(*infoAOs_, *hcore_, *Pmatrix, all2CIntegral_);
  return Pmatrix->Alloc4Matrix("Pmatrix") && Fmatrix->Alloc4Matrix("Fmatrix");
}

bool SCFCalculation::DeallocSCFData() {
  delete[] eigenVec;
  delete[] eigenVal;
  eigenVec = eigenVal = nullptr;
  if (Pmatrix) { Pmatrix->Dealloc4Matrix(); delete Pmatrix; Pmatrix = nullptr; }
  if (Fmatrix) { Fmatrix->Dealloc4Matrix(); delete Fmatrix; Fmatrix = nullptr; }
  return true;
}

// The whole loop of scfcalculation.cpp:66-146 runs on the device; the step lines are printed
// afterwards from the energy history.  The per-stage millisecond fields of the reference's
// line are reported as 0 and StepTime as the mean device step time.
void SCFCalculation::ComputeSCF() {
  sgb_mol* m = infoAOs_->device();
  if (!m) return;
  sgb_scf_result r{};
  stepEnergies.assign(maxSCFSteps + 1, 0.0);
  const auto t0 = std::chrono::high_resolution_clock::now();
  const int rc = sgb_scf(semigpu::context(), m, thresholdEnergy, (int)maxSCFSteps, &r,
                         stepEnergies.data());
  const auto t1 = std::chrono::high_resolution_clock::now();
  if (rc < 0) {
    check(rc, "sgb_scf");
    return;
  }
  stepEnergies.resize(r.n_iter + 1);
  SCFSteps = r.n_iter;
  const long step_ms =
      r.n_iter ? (long)(std::chrono::duration<double, std::milli>(t1 - t0).count() / r.n_iter) : 0;
  cout << "SCF step : " << 0 << "  Energy = " << stepEnergies[0] << endl;
  for (int k = 1; k <= r.n_iter; ++k) {
    cout << "SCF step : " << k;
    cout << "  Energy = " << stepEnergies[k];
    cout << "  LapackTime = " << 0;
    cout << "  PmatTime = " << 0;
    cout << "  FmatTime = " << 0;
    cout << "  EnerTime = " << 0;
    cout << "  StepTime = " << step_ms << endl;
  }
  if (rc == SGB_E_EIG) cout << "LAPACK: The algorithm failed to converge" << endl;
  finalEnergy = r.e_el;
  energyConverge = r.converged != 0;
  sgb_ctx* c = semigpu::context();
  check(sgb_get(c, m, SGB_EIGVEC, eigenVec, nAOs_ * nAOs_), "sgb_get");
  check(sgb_get(c, m, SGB_EIGVAL, eigenVal, nAOs_), "sgb_get");
  if (Pmatrix && Pmatrix->matrixHold_)
    check(sgb_get(c, m, SGB_DENSITY, Pmatrix->matrixHold_, Pmatrix->array1DSize_), "sgb_get");
  if (Fmatrix && Fmatrix->matrixHold_)
    check(sgb_get(c, m, SGB_FOCK, Fmatrix->matrixHold_, Fmatrix->array1DSize_), "sgb_get");
}

double CoreCoreRepulsion::ComputeRepulsion(const MNDOparameter&, const ListAtomicOrbitals& infoAOs,
                                           double****) {
  sgb_mol* m = infoAOs.device();
  double e = 0.0;
  if (m) check(sgb_core_core(semigpu::context(), m, &e), "sgb_core_core");
  return e;
}

void ScreenUtils::PrintScrStarLine(void) {
  for (int i = 0; i < 80; ++i) std::cout << '*';
  std::cout << std::endl;
}
