// RunIAC.h -- the evaluation pipeline of FabianTr/IncohAutoCorrelate
// (IAC/RunIAC.h, IAC/RunIAC.cpp:120-632) and the settings loaders of its run
// modes (IAC/MainRunModes.cpp:32-91, :246-328) over the classes of this
// library.  Frames are read through Settings::Frames; pixel maps, masks and
// outputs are raw binary files (HDF5 is not part of this build):
//   PixelMap_Path     float32 [ss][fs][3], PixelMap_DataSet = "ss,fs" (its shape)
//   PixelMask_Path    int32 [ss][fs] ("" = all ones)
//   outputs           float64 arrays as the reference's SafeArrayToFile(Binary)
#pragma once

#include <string>

#include "AC1D.h"
#include "Detector.h"
#include "Simulator.h"

namespace iac {
namespace RunIAC {

struct IAC_Report {
    double dQperVox = 0;
    unsigned int FinalMeshSize = 0;
    unsigned int SmallCqMeshSize[3] = {0, 0, 0};
    unsigned int LowerBound = 0, UpperBound = 0;
    float MeanPhotonCount = 0;
    unsigned long long PhotonPairs = 0;
    double Seconds = 0;
};

struct CreateDataEval_Settings {
    std::string PixelMap_Path, PixelMap_DataSet, PixelMask_Path, PixelMask_Dataset, XML_Path;
    bool UseExistingAvInt = false;
    std::string Out_Final_AC_Path, Out_AvIntensity_Path, Out_Cq_Path, Out_Cq_small_Path, Out_ACuw_Path,
        Out_Q_Vector, Out_Report;
    int MeshSize = 201;
    float QZoom = 1.0f;
    bool AngularAveraged = false;
    bool DoubleMap = true;
    Detector::AutoCorrFlags AC_FirstMap_Flags{Settings::NearestNeighbour};
    Detector::AutoCorrFlags AC_SecondMap_Flags{Settings::NearestNeighbour};
    float PhotonOffset = 0.0f, PhotonStep = 1.0f;
    bool RestrictStackToBoundaries = false;
    unsigned int LowerBoundary = 0, UpperBoundary = 10;
    bool UsePixelMask_as_Flatfield = false;
    bool InvertRotMatrix = false;
    bool IgnoreOrientation = false;
    int EchoLevel = 3;
};

IAC_Report Run_AutoCorr_DataEval(Settings &PrgSettings, CreateDataEval_Settings EvalSettings);
void Merge_ACandCQ(double *&Output, ACMesh &AC, ACMesh &CQ, Settings &PrgSettings);
void Merge_ACandCQ(double *&Output, double *AC, ACMesh &CQ, Settings &PrgSettings);

CreateDataEval_Settings LoadEvaluationSettings(std::string Filename, Settings &Options);

struct AllSimSettings {
    Simulator::SimulationSettings SimSettings;
    double LatticeVector[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    unsigned int UnitCells[3] = {10, 10, 10};
    std::vector<std::array<double, 3>> UnitCell;
    std::string PixelMap_Path, PixelMap_DataSet;
};
AllSimSettings LoadSimulationSettings(std::string Filename, Settings &Options);

void SafeArrayToFile(const std::string &path, const double *a, size_t n);
void SafeArrayToFile(const std::string &path, const float *a, size_t n);
void LoadPixelMapFile(Detector &Det, const std::string &path, const std::string &shape);

}  // namespace RunIAC
}  // namespace iac
