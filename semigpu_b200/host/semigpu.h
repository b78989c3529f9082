// C++ host API with the reference's class names and signatures (LuisAlfredoNu/semiGPU,
// src/common/*.h), implemented over the C ABI of include/semigpu_b200.h.  Code written against
// the reference's stage API (src/App/semiGPU.cc:29-104) compiles against this header and runs
// every stage on the GPU.
//
// What stays on the host is what the reference keeps there as data: the atom list, the AO
// table, the ragged integral array mirrored back for GetValueFromArray, and the matrices'
// matrixHold_ copies.  Every number in them is computed by the CUDA library.  The device
// molecule behind a ListAtomicOrbitals is created by ComputeAllTwoCenterIntegral and reused by
// Hcore, SCFCalculation and CoreCoreRepulsion.
#ifndef SEMIGPU_B200_HOST_H
#define SEMIGPU_B200_HOST_H

#include <string>
#include <vector>

using std::string;
using std::vector;

struct sgb_mol;
struct sgb_ctx;

// ---- atom.h -----------------------------------------------------------------------------
class Atom {
 public:
  Atom();
  int atomNumber;
  string atomSymbol;
  double atomCoordinates[3];
  double atomWeight;
  int atomValenceElectrons;
  bool statusData;
  void setCoordinates(double, double, double);
  void setCoordinates(vector<double>);
  void setCoordinates(double (&xyz)[3]);
  double getXCoordinate();
  double getYCoordinate();
  double getZCoordinate();
  void setAtomSymbol(string);
  void setAtomNumber(int);
  static void PrintGeometry(const vector<Atom>& molecule);
};

// ---- readxyzfile.h ----------------------------------------------------------------------
class ReadXYZFile {
 public:
  ReadXYZFile();
  int Natoms;
  bool open_without_problems;
  bool GetValuesFromFile(string, vector<Atom>&);
  // Every frame of a multi-frame XYZ file (blocks of count line, comment line, atoms, one after
  // the other; blank lines between blocks allowed) with its comment line.  Not in the reference.
  bool GetFramesFromFile(string, vector<vector<Atom>>&, vector<string>&);
};

// ---- atomicOrbitals.h -------------------------------------------------------------------
class AtomicOrbital {
 public:
  AtomicOrbital();
  int indexAtom;
  int element;
  int angularMomentum[3];
  int angularMomentumInt;
  int indexAO;
  double coordinates[3];  // bohr
  int GetCoreCharge() const;
  int GetAOsSize() const;
};

class ListAtomicOrbitals {
 public:
  ListAtomicOrbitals();
  ~ListAtomicOrbitals();
  AtomicOrbital* orbital;
  bool statusData;
  void SetOrbitals(const vector<Atom>&);
  size_t size() const;
  // engine side: the atoms this list was built from and its device molecule
  vector<int> Z;
  vector<double> xyz;  // Angstrom
  sgb_mol* device() const;

 private:
  size_t totalOrbitals_;
  mutable sgb_mol* mol_;
};

// ---- MNDO_parameters.h ------------------------------------------------------------------
class MNDOparameter {
 public:
  MNDOparameter();
  ~MNDOparameter();
  unsigned int countParameter_;
  double *uss, *upp, *zs, *betaS, *betaP, *alpha, *gss, *gpp, *gsp, *gp2, *hsp;
  double **dd;  // [2]
  double **pp;  // [3]
  double *heat, *eisol;
};

// ---- twocenterintegral.h ----------------------------------------------------------------
class TwoCenterIntegral {
 public:
  TwoCenterIntegral(MNDOparameter&);
  static bool Alloc4AllTwoCenterIntegral(const vector<Atom>& molecule, double****& ints);
  static bool Dealloc4AllTwoCenterIntegral(const vector<Atom>& molecule, double****& ints);
  void ComputeAllTwoCenterIntegral(const ListAtomicOrbitals& infoAOs, double****& ints);
  static double GetValueFromArray(const AtomicOrbital&, const AtomicOrbital&,
                                  const AtomicOrbital&, const AtomicOrbital&, double**** ints);
  static void To_device(const vector<Atom>& molecule, double****& ints);

 private:
  MNDOparameter* parameter;
};

// ---- basematrix.h -----------------------------------------------------------------------
class BaseMatrix {
 public:
  BaseMatrix();
  explicit BaseMatrix(size_t);
  virtual ~BaseMatrix();
  size_t matrixSize_;
  double* matrixHold_;
  size_t array1DSize_;
  bool Alloc4Matrix(string matrixName);
  bool Dealloc4Matrix();
  virtual void ComputeMatrix();
};

// ---- hcore.h ----------------------------------------------------------------------------
class Hcore : public BaseMatrix {
 public:
  Hcore(const MNDOparameter&, const ListAtomicOrbitals&, double****);
  void ComputeMatrix() override;

 private:
  const ListAtomicOrbitals* infoAOs_;
};

// ---- densitymatrix.h / fockmatrix.h -----------------------------------------------------
class DensityMatrix : public BaseMatrix {
 public:
  DensityMatrix(const ListAtomicOrbitals& infoAOs, const double* eigenVec, const size_t nAOs);
  void GuessDensityMatrixSwitch(bool);
  // guess mode: P_ii = Z_A / nAO_A (densitymatrix.cpp:26-37); otherwise the density of the
  // molecule's last device SCF step
  void ComputeMatrix() override;

 private:
  const ListAtomicOrbitals* infoAOs_;
  bool guessSwitch_;
};

class FockMatrix : public BaseMatrix {
 public:
  FockMatrix(const ListAtomicOrbitals&, const Hcore&, const DensityMatrix&, double****&);
  // F = Hcore + G(P) on the device for the current Pmatrix contents (fockmatrix.cpp:32-53)
  void ComputeMatrix() override;
  double lastElectronicEnergy;

 private:
  const ListAtomicOrbitals* infoAOs_;
  const DensityMatrix* Pmatrix_;
};

// ---- electronicenergy.h -----------------------------------------------------------------
class ElectronicEnergy {
 public:
  ElectronicEnergy();
  // 1/2 sum_ij P_ij (H_ij + F_ij) of the three matrixHold_ arrays (electronicenergy.cpp:12-36),
  // reduced on the device
  static double ComputeEnergy(const size_t& nAOs, const Hcore&, const FockMatrix&,
                              const DensityMatrix&);
};

// ---- scfcalculation.h -------------------------------------------------------------------
class SCFCalculation {
 public:
  SCFCalculation(const ListAtomicOrbitals&, double****&, const Hcore&);
  double* eigenVec;  // nAOs x nAOs, column-major, column k = eigenvector k
  double* eigenVal;
  DensityMatrix* Pmatrix;
  FockMatrix* Fmatrix;
  double finalEnergy;
  bool energyConverge;
  // The reference hard-codes 5e-3 eV and 100 steps (scfcalculation.cpp:74-77); both are
  // settable here, with the same defaults.
  double thresholdEnergy;
  unsigned int maxSCFSteps;
  unsigned int SCFSteps;
  vector<double> stepEnergies;
  bool AllocSCFData();
  bool DeallocSCFData();
  void ComputeSCF();

 private:
  const ListAtomicOrbitals* infoAOs_;
  size_t nAOs_;
  double**** all2CIntegral_;
  const Hcore* hcore_;
};

// ---- corecorerepulsion.h ----------------------------------------------------------------
class CoreCoreRepulsion {
 public:
  static double ComputeRepulsion(const MNDOparameter&, const ListAtomicOrbitals&, double****);
};

// ---- screenutils.h (the part the CLI prints) ---------------------------------------------
class ScreenUtils {
 public:
  static void PrintScrStarLine(void);
};

// ---- engine access -----------------------------------------------------------------------
namespace semigpu {
// The process-wide context (device from SEMIGPU_DEVICE, default 0); created on first use.
sgb_ctx* context();
// Status of the last failed engine call (0 if none) and its message.
int last_status();
const char* last_error();
}  // namespace semigpu

#endif  // SEMIGPU_B200_HOST_H
