// RunIAC.cpp -- evaluation pipeline and run-mode settings over this library
// (IAC/RunIAC.cpp:120-632, IAC/MainRunModes.cpp:32-91, :246-328).
#include "RunIAC.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include "PropertyTree.h"

namespace iac {
namespace RunIAC {

void SafeArrayToFile(const std::string &path, const double *a, size_t n)
{
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    const size_t w = std::fwrite(a, sizeof(double), n, f);
    std::fclose(f);
    if (w != n) throw std::runtime_error("short write to " + path);
}

void SafeArrayToFile(const std::string &path, const float *a, size_t n)
{
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    const size_t w = std::fwrite(a, sizeof(float), n, f);
    std::fclose(f);
    if (w != n) throw std::runtime_error("short write to " + path);
}

static std::vector<char> read_file(const std::string &path, size_t bytes)
{
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<char> b(bytes);
    const size_t r = std::fread(b.data(), 1, bytes, f);
    std::fclose(f);
    if (r != bytes) throw std::runtime_error(path + " is shorter than " + std::to_string(bytes) + " bytes");
    return b;
}

void LoadPixelMapFile(Detector &Det, const std::string &path, const std::string &shape)
{
    unsigned ss = 0, fs = 0;
    char sep = 0;
    std::istringstream is(shape);
    if (!(is >> ss >> sep >> fs) || ss == 0 || fs == 0)
        throw std::runtime_error("PixelMap_Dataset must give the map's shape as \"ss,fs\" (got \"" + shape + "\")");
    const auto b = read_file(path, (size_t)ss * fs * 3 * sizeof(float));
    Det.LoadPixelMap(reinterpret_cast<const float *>(b.data()), ss, fs);
}

// IAC/RunIAC.cpp:120-158
void Merge_ACandCQ(double *&Output, ACMesh &AC, ACMesh &CQ, Settings &S)
{
    const size_t n = (size_t)AC.Shape.Size_AB * AC.Shape.Size_AB * AC.Shape.Size_C;
    std::vector<double> ac(n);
    for (size_t i = 0; i < n; i++) ac[i] = S.IntToFloat(AC.Mesh[i]);
    Merge_ACandCQ(Output, ac.data(), CQ, S);
}

void Merge_ACandCQ(double *&Output, double *AC, ACMesh &CQ, Settings &)
{
    const size_t n = (size_t)CQ.Shape.Size_AB * CQ.Shape.Size_AB * CQ.Shape.Size_C;
    Output = new double[n]();
    for (size_t i = 0; i < n; i++) {
        Output[i] = CQ.CQMesh[i] <= 0 ? 0.0 : AC[i] / CQ.CQMesh[i];
        if (std::isnan(Output[i])) Output[i] = 0;
    }
}

// IAC/RunIAC.cpp:185-632
IAC_Report Run_AutoCorr_DataEval(Settings &P, CreateDataEval_Settings E)
{
    const auto t0 = std::chrono::steady_clock::now();
    IAC_Report R;
    Detector Det;
    if (E.PixelMap_Path.empty()) throw std::runtime_error("No pixel map path set => can't load Hit Events");
    LoadPixelMapFile(Det, E.PixelMap_Path, E.PixelMap_DataSet);
    Det.Calc_kMap();
    if (E.PixelMask_Path.empty()) {
        Det.GenerateFlatOnesPixelMask();
    } else {
        const auto b = read_file(E.PixelMask_Path, Det.Pixels() * sizeof(int));
        Det.LoadPixelMask(reinterpret_cast<const int *>(b.data()));
    }
    if (E.XML_Path.empty()) throw std::runtime_error("No XML path set => can't load Hit Events");
    P.LoadHitEventListFromFile(E.XML_Path);
    if (E.InvertRotMatrix) P.InvertRotationMatrices();
    unsigned lower = 0, upper = (unsigned)P.HitEvents.size();
    if (E.RestrictStackToBoundaries) {
        if (E.UpperBoundary > P.HitEvents.size())
            throw std::runtime_error("Upper Hit boundary exeeds number of hits in loaded XML file");
        lower = E.LowerBoundary;
        upper = E.UpperBoundary;
    }
    R.LowerBound = lower;
    R.UpperBound = upper;
    if (E.IgnoreOrientation)
        for (auto &ev : P.HitEvents) {
            const float id[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
            std::copy(id, id + 9, ev.RotMatrix);
        }
    // averaged intensity (flat field), IAC/RunIAC.cpp:303-340
    const size_t npix = Det.Pixels();
    if (E.UseExistingAvInt && !E.UsePixelMask_as_Flatfield) {
        const auto b = read_file(E.Out_AvIntensity_Path, npix * sizeof(float));
        std::copy(reinterpret_cast<const float *>(b.data()), reinterpret_cast<const float *>(b.data()) + npix,
                  Det.Intensity);
        Det.ApplyPixelMask();
    } else if (!E.UsePixelMask_as_Flatfield) {
        Det.LoadAndAverageIntensity(P.HitEvents, E.PhotonOffset, E.PhotonStep, (int)lower, (int)upper, true, P);
        if (!E.Out_AvIntensity_Path.empty()) SafeArrayToFile(E.Out_AvIntensity_Path, Det.Intensity, npix);
        Det.ApplyPixelMask();
    } else {
        for (size_t i = 0; i < npix; i++) Det.Intensity[i] = (float)Det.PixelMask[i];
        Det.Checklist.Intensity = true;
    }

    if (E.AngularAveraged) {  // 1D, IAC/RunIAC.cpp:342-439 (interpolation fixed to linear)
        const Settings::Interpolation interp = Settings::Linear;
        AC1D V;
        V.Initialize(Det, (unsigned)E.MeshSize, E.QZoom);
        V.Calculate_CQ(Det, P, interp);
        if (!E.Out_Cq_Path.empty()) SafeArrayToFile(E.Out_Cq_Path, V.CQ, V.Shape.Size);
        V.Calculate_AC_UW_MR(P, Det, interp, {E.PhotonOffset, E.PhotonStep}, lower, upper);
        if (!E.Out_ACuw_Path.empty()) SafeArrayToFile(E.Out_ACuw_Path, V.AC_UW, V.Shape.Size);
        V.CalcAC();
        if (!E.Out_Final_AC_Path.empty()) SafeArrayToFile(E.Out_Final_AC_Path, V.AC, V.Shape.Size);
        if (!E.Out_Q_Vector.empty()) {
            V.CreateQVector();
            SafeArrayToFile(E.Out_Q_Vector, V.Q, V.Shape.Size);
        }
        R.dQperVox = V.Shape.dq_per_Step;
        R.FinalMeshSize = V.Shape.Size;
    } else {  // 3D, IAC/RunIAC.cpp:440-626
        ACMesh small(&P), CQ(&P), AC(&P);
        small.CreateSmallMesh_CofQ_ForDetector(Det, E.MeshSize, E.QZoom);
        Det.AutoCorrelate_CofQ_SmallMesh(small, E.AC_FirstMap_Flags, P);
        const size_t sn = (size_t)small.Shape.Size_AB * small.Shape.Size_AB * small.Shape.Size_C;
        if (!E.Out_Cq_small_Path.empty()) SafeArrayToFile(E.Out_Cq_small_Path, small.CQMesh, sn);
        CQ.CreateBigMesh_CofQ_ForDetector(Det, E.MeshSize, E.QZoom);
        Det.Merge_smallCofQ(CQ, small, P.HitEvents, lower, upper, P, E.AC_SecondMap_Flags);
        const size_t bn = (size_t)CQ.Shape.Size_AB * CQ.Shape.Size_AB * CQ.Shape.Size_C;
        if (!E.Out_Cq_Path.empty()) SafeArrayToFile(E.Out_Cq_Path, CQ.CQMesh, bn);
        AC.CreateBigMeshForDetector(Det, E.MeshSize, E.QZoom);
        for (unsigned i = lower; i < upper; i++) {  // the per-frame loop, IAC/RunIAC.cpp:524-550
            Det.LoadIntensityData(&P.HitEvents[i], P);
            R.MeanPhotonCount += P.HitEvents[i].PhotonCount;
            Det.ApplyPixelMask();
            Det.CreateSparseHitList(E.PhotonOffset, E.PhotonStep);
            const unsigned long long n = Det.SparseHitList.size();
            R.PhotonPairs += n * (n + 1) / 2;
            Det.AutoCorrelateSparseList(AC, E.AC_FirstMap_Flags, E.AC_SecondMap_Flags, E.DoubleMap, P);
        }
        AC.Sync(P);
        R.MeanPhotonCount = R.MeanPhotonCount / ((float)(upper - lower));
        if (!E.Out_ACuw_Path.empty()) {
            std::vector<double> m(bn);
            for (size_t i = 0; i < bn; i++) m[i] = P.IntToFloat(AC.Mesh[i]);
            SafeArrayToFile(E.Out_ACuw_Path, m.data(), bn);
        }
        double *final_ac = nullptr;
        Merge_ACandCQ(final_ac, AC, CQ, P);
        if (!E.Out_Final_AC_Path.empty()) SafeArrayToFile(E.Out_Final_AC_Path, final_ac, bn);
        delete[] final_ac;
        R.dQperVox = AC.Shape.dq_per_Voxel;
        R.FinalMeshSize = AC.Shape.Size_AB;
        R.SmallCqMeshSize[0] = small.Shape.Size_AB;
        R.SmallCqMeshSize[1] = small.Shape.Size_AB;
        R.SmallCqMeshSize[2] = small.Shape.Size_C;
    }
    R.Seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (!E.Out_Report.empty()) {
        std::FILE *f = std::fopen(E.Out_Report.c_str(), "w");
        if (f) {
            std::fprintf(f, "IAC report\nevents %u..%u\nmesh %u\ndq per voxel %.9g\nsmall C(q) %u x %u x %u\n"
                            "mean photon count %.6g\nphoton pairs %llu\nseconds %.3f\n",
                         R.LowerBound, R.UpperBound, R.FinalMeshSize, R.dQperVox, R.SmallCqMeshSize[0],
                         R.SmallCqMeshSize[1], R.SmallCqMeshSize[2], R.MeanPhotonCount, R.PhotonPairs, R.Seconds);
            std::fclose(f);
        }
    }
    return R;
}

// IAC/MainRunModes.cpp:32-91
CreateDataEval_Settings LoadEvaluationSettings(std::string Filename, Settings &Options)
{
    const PropertyTree pt = PropertyTree::ReadXml(Filename);
    CreateDataEval_Settings E;
    const std::string b = "root.EvalSettings.";
    E.XML_Path = pt.Get(b + "InputFiles.EventList_Path", std::string());
    E.PixelMap_Path = pt.Get(b + "InputFiles.PixelMap_Path", std::string());
    E.PixelMap_DataSet = pt.Get(b + "InputFiles.PixelMap_Dataset", std::string());
    E.PixelMask_Path = pt.Get(b + "InputFiles.PixelMask_Path", std::string());
    E.PixelMask_Dataset = pt.Get(b + "InputFiles.PixelMask_Dataset", std::string());
    E.UseExistingAvInt = pt.GetBool(b + "InputFiles.UseExistingAvInt", false);
    E.Out_Final_AC_Path = pt.Get(b + "OutputFiles.AC_Final_Path", std::string());
    E.Out_AvIntensity_Path = pt.Get(b + "OutputFiles.AvIntensity_Path", std::string());
    E.Out_Cq_Path = pt.Get(b + "OutputFiles.Cq_Merged_Path", std::string());
    E.Out_Cq_small_Path = pt.Get(b + "OutputFiles.Cq_small_Path", std::string());
    E.Out_ACuw_Path = pt.Get(b + "OutputFiles.ACuw_Path", std::string());
    E.Out_Q_Vector = pt.Get(b + "OutputFiles.Q_Vector", std::string());
    E.MeshSize = pt.Get<int>(b + "OutputMesh.MeshSize", 201);
    E.QZoom = pt.Get<float>(b + "OutputMesh.QZoom", 1.0f);
    E.AngularAveraged = pt.GetBool(b + "OutputMesh.AngularAveraged", false);
    E.DoubleMap = pt.GetBool(b + "OutputMesh.DoubleMap", true);
    E.AC_FirstMap_Flags.InterpolationMode =
        (Settings::Interpolation)pt.Get<int>(b + "OutputMesh.AC_FirstMap_Flags.InterpolationMode", 0);
    E.AC_SecondMap_Flags.InterpolationMode =
        (Settings::Interpolation)pt.Get<int>(b + "OutputMesh.AC_SecondMap_Flags.InterpolationMode", 0);
    E.PhotonOffset = pt.Get<float>(b + "PhotonThreshold.PhotonOffset", 0.0f);
    E.PhotonStep = pt.Get<float>(b + "PhotonThreshold.PhotonStep", 1.0f);
    E.RestrictStackToBoundaries = pt.GetBool(b + "Misc.RestrictStackToBoundaries", false);
    E.LowerBoundary = pt.Get<unsigned>(b + "Misc.LowerBoundary", 0u);
    E.UpperBoundary = pt.Get<unsigned>(b + "Misc.UpperBoundary", 10u);
    E.UsePixelMask_as_Flatfield = pt.GetBool(b + "Misc.UsePixelmaskAsFlatField", false);
    E.InvertRotMatrix = pt.GetBool(b + "Misc.InvertRotMatrix", false);
    E.EchoLevel = pt.Get<int>(b + "Misc.EchoLevel", 3);
    E.Out_Report = pt.Get(b + "Misc.Report_Path", std::string());
    if (E.EchoLevel == 0) Options.echo = false;
    return E;
}

static void split3(const std::string &s, double *out, int n)
{
    std::string in = s;
    for (int i = 0; i < n; i++) {
        const size_t p = in.find(';');
        out[i] = std::atof(in.substr(0, p).c_str());
        if (p == std::string::npos) {
            if (i != n - 1) throw std::runtime_error("expected " + std::to_string(n) + " values in \"" + s + "\"");
            return;
        }
        in.erase(0, p + 1);
    }
}

// IAC/MainRunModes.cpp:246-328 (the simulation part)
AllSimSettings LoadSimulationSettings(std::string Filename, Settings &)
{
    const PropertyTree pt = PropertyTree::ReadXml(Filename);
    AllSimSettings A;
    auto &S = A.SimSettings;
    const std::string b = "root.Simulation.";
    S.Filename_XML = pt.Get(b + "OutputPath_EventList", std::string("SimOut.xml"));
    S.Filename_Intensity = pt.Get(b + "OutputPath_Intensities", std::string("SimOut.raw"));
    S.Dataset = pt.Get(b + "OutputDataset_Intensities", std::string("data"));
    S.SaveResults = pt.GetBool(b + "SaveResults", true);
    S.Wavelength = pt.Get<double>(b + "Wavelength", 1.94);
    S.NumberOfSimulations = pt.Get<unsigned>(b + "NumberOfPattern", 10u);
    S.Modes = pt.Get<unsigned>(b + "NumberOfModes", 1u);
    S.CrystSettings.FlYield = pt.Get<float>(b + "FluorescenceYield", 1.0f);
    S.CrystSettings.Incoherent = pt.GetBool(b + "Incoherent", true);
    S.CrystSettings.RandOrientation = pt.GetBool(b + "RandomOriented", false);
    S.CrystSettings.Isotropie = pt.Get<float>(b + "OrientationIsotropie", 1.0f);
    S.AveragePhotonesPerEmitterOnDetector = pt.Get<float>(b + "AveragePhotonesPerEmitterOnDetector", 1.0f);
    S.SubSampling = pt.Get<unsigned>(b + "SubSampling", 1u);
    S.PoissonSample = pt.GetBool(b + "PoissonSample", true);
    S.Value_per_Photon = pt.Get<float>(b + "ValuePerPhoton", 1.0f);
    S.ADUNoise = pt.Get<float>(b + "ADUNoise", 0.0f);
    S.AutoPixelOrientation = pt.GetBool(b + "AutoPixelOrientation", true);
    S.AutoPixelSize = pt.GetBool(b + "AutoPixelSize", true);
    S.IntensitySquared = pt.GetBool(b + "IntensitySquared", false);
    S.Seed = pt.Get<unsigned long long>(b + "Seed", 0ull);
    split3(pt.Get(b + "PixelOrientationVectors", std::string("0.0; 1.0; 0.0; 0.0; 0.0; 1.0")),
           S.PixelOrientationVectors, 6);
    split3(pt.Get(b + "PixelSize", std::string("50.0; 50.0")), S.PixelSize, 2);
    double uc[3];
    split3(pt.Get(b + "UnitCells", std::string("10; 10; 10")), uc, 3);
    for (int d = 0; d < 3; d++) A.UnitCells[d] = (unsigned)uc[d];
    for (int k = 0; k < 3; k++) {
        const char *def[3] = {"1.0; 0.0; 0.0", "0.0; 1.0; 0.0", "0.0; 0.0; 1.0"};
        split3(pt.Get(b + "LatticeVector_" + std::to_string(k + 1), std::string(def[k])), A.LatticeVector[k], 3);
    }
    const unsigned noe = pt.Get<unsigned>(b + "UnitCell.NumberOfEmittersPerUnitcell", 0u);
    for (unsigned i = 0; i < noe; i++) {
        std::array<double, 3> e;
        split3(pt.Get(b + "UnitCell.Emitter_" + std::to_string(i + 1), std::string("0.0; 0.0; 0.0")), e.data(), 3);
        A.UnitCell.push_back(e);
    }
    A.PixelMap_Path = pt.Get(b + "PixelMap_Path", std::string());
    A.PixelMap_DataSet = pt.Get(b + "PixelMap_Dataset", std::string());
    return A;
}

}  // namespace RunIAC
}  // namespace iac
