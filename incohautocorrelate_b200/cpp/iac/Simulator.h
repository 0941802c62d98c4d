// Simulator.h -- Crystal and Simulator of FabianTr/IncohAutoCorrelate
// (IAC/Crystal.h, IAC/Simulator.h) over libiac_b200: emitters, emitter-phase
// intensities, photon statistics on the device, frame by frame in batches.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "Detector.h"

namespace iac {

class Crystal {
public:
    // IAC/Crystal.cpp:7-13, :192-229: a lattice of CrystalSize cells centred at
    // the origin with the unit cell's emitters in each cell
    Crystal(double LatticeVector[3][3], unsigned int CrystalSize[3], std::vector<std::array<double, 3>> UnitCell);

    std::vector<std::array<double, 3>> AtomPositions;

    struct EmittingCrystSettings {
        bool Incoherent = true;
        float FlYield = 1.0f;
        bool RandOrientation = false;
        float Isotropie = 1.0f;
    };
};

class Simulator {
public:
    struct SimulationSettings {
        double Wavelength = 1.94;
        unsigned int NumberOfSimulations = 10;
        unsigned int Modes = 1;
        Crystal::EmittingCrystSettings CrystSettings;
        float AveragePhotonesPerEmitterOnDetector = 1.0f;
        unsigned int SubSampling = 1;
        bool PoissonSample = true;
        float Value_per_Photon = 1.0f;
        float ADUNoise = 0.0f;
        bool AutoPixelOrientation = true;
        bool AutoPixelSize = true;
        double PixelOrientationVectors[6] = {0, 1, 0, 0, 0, 1};
        double PixelSize[2] = {50, 50};
        std::string Filename_Intensity = "SimOut.raw";
        std::string Dataset = "data";
        std::string Filename_XML = "SimOut.xml";
        bool SaveResults = false;
        // emitter-phase sum per sub-pixel: |Psi| as the reference's kernel adds
        // (IAC/kernel.cl:844) or |Psi|^2
        bool IntensitySquared = false;
        uint64_t Seed = 0;  // 0: draw one from std::random_device
        unsigned int FramesPerLaunch = 512;
    };

    struct SimulationOutput {
        std::vector<std::vector<float>> Intensities;
        std::vector<Settings::HitEvent> HitEvents;
        unsigned int DetectorSize[2] = {0, 0};
    };

    // IAC/Simulator.cpp:1248-1392 (the two host threads become device batches)
    void ParSimulate(Crystal EmitterCrystal, Detector &Det, SimulationSettings SimSettings,
                     SimulationOutput &Output, Settings &Options);
    // IAC/Simulator.cpp:415-488 with HDF5 replaced by a raw float32 stack
    static void SaveSimulationOutput(SimulationOutput &Output, std::string Filename_Intensity,
                                     std::string Filename_XML, SimulationSettings SimSettings, Settings &Options);
    // IAC/Simulator.cpp:495-519
    static void GeneratePixelMap(int SizeA, int SizeB, float PixelSize, std::array<float, 3> Center,
                                 std::array<float, 3> VecA, std::array<float, 3> VecB, std::vector<float> &PixelMap);
};

}  // namespace iac
