// iac_run -- command-line driver of the evaluation and simulation run modes
// (IAC/main.cpp:560-573 "-e", :852-865 "-s"; IAC/MainRunModes.cpp:1254-1326,
// :1478-1518) over libiac_b200.
//
//   iac_run -e EvalSettings.xml [device]   3D or angular-averaged evaluation
//   iac_run -s SimSettings.xml  [device]   simulate frames to a raw stack + XML event list
//
// Settings files use the reference's keys (root.EvalSettings.*, root.Simulation.*);
// pixel maps, masks and frame stacks are raw binary files (see RunIAC.h).
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <iostream>
#include <string>

#include "iac/RunIAC.h"

using namespace iac;

static int evaluate(const std::string &file, int device)
{
    Settings S;
    S.SetUp_Device(device);
    S.Frames = std::make_shared<RawStackSource>();
    RunIAC::CreateDataEval_Settings E = RunIAC::LoadEvaluationSettings(file, S);
    const RunIAC::IAC_Report R = RunIAC::Run_AutoCorr_DataEval(S, E);
    std::printf("{\"mode\": \"evaluate\", \"mesh\": %u, \"events\": %u, \"photon_pairs\": %llu, "
                "\"seconds\": %.4f, \"dq_per_voxel\": %.9g}\n",
                R.FinalMeshSize, R.UpperBound - R.LowerBound, R.PhotonPairs, R.Seconds, R.dQperVox);
    return 0;
}

static int simulate(const std::string &file, int device)
{
    Settings S;
    S.SetUp_Device(device);
    RunIAC::AllSimSettings A = RunIAC::LoadSimulationSettings(file, S);
    if (A.PixelMap_Path.empty()) throw std::runtime_error("root.Simulation.PixelMap_Path is required");
    Detector Det;
    RunIAC::LoadPixelMapFile(Det, A.PixelMap_Path, A.PixelMap_DataSet);
    if (A.UnitCell.empty()) A.UnitCell.push_back({0.0, 0.0, 0.0});
    Crystal C(A.LatticeVector, A.UnitCells, A.UnitCell);
    Simulator Sim;
    Simulator::SimulationOutput Out;
    A.SimSettings.SaveResults = true;
    Sim.ParSimulate(C, Det, A.SimSettings, Out, S);
    std::printf("{\"mode\": \"simulate\", \"frames\": %zu, \"emitters\": %zu, \"stack\": \"%s\", \"events\": \"%s\"}\n",
                Out.Intensities.size(), C.AtomPositions.size(), A.SimSettings.Filename_Intensity.c_str(),
                A.SimSettings.Filename_XML.c_str());
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s -e|-s settings.xml [device]\n", argv[0]);
        return 2;
    }
    const std::string mode = argv[1], file = argv[2];
    const int device = argc > 3 ? std::atoi(argv[3]) : 0;
    try {
        if (mode == "-e") return evaluate(file, device);
        if (mode == "-s") return simulate(file, device);
        std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
        return 2;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "iac_run: %s\n", e.what());
        return 1;
    }
}
