// Simulator.cpp -- Crystal and Simulator over libiac_b200
// (IAC/Crystal.cpp, IAC/Simulator.cpp:415-944, :1248-1392).
#include "Simulator.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <stdexcept>

namespace iac {

Crystal::Crystal(double LV[3][3], unsigned int CS[3], std::vector<std::array<double, 3>> UnitCell)
{
    const unsigned l = CS[0], m = CS[1], n = CS[2];
    std::vector<std::array<double, 3>> lattice((size_t)l * m * n);
    for (unsigned x = 0; x < l; x++)
        for (unsigned y = 0; y < m; y++)
            for (unsigned z = 0; z < n; z++)
                for (int d = 0; d < 3; d++)
                    lattice[z + (size_t)n * y + (size_t)n * m * x][d] = (x - l / 2.0 + 0.5) * LV[0][d] +
                                                                         (y - m / 2.0 + 0.5) * LV[1][d] +
                                                                         (z - n / 2.0 + 0.5) * LV[2][d];
    const size_t k = UnitCell.size();
    AtomPositions.resize(lattice.size() * k);
    for (size_t i = 0; i < lattice.size(); i++)
        for (size_t j = 0; j < k; j++)
            for (int d = 0; d < 3; d++) AtomPositions[i * k + j][d] = lattice[i][d] + UnitCell[j][d];
}

namespace {
struct DevBuf {
    iac_ctx *ctx = nullptr;
    void *p = nullptr;
    DevBuf(iac_ctx *c, size_t bytes) : ctx(c) { Check(iac_device_alloc(c, std::max<size_t>(bytes, 16), &p), "iac_device_alloc"); }
    ~DevBuf()
    {
        if (p) iac_device_free(ctx, p);
    }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};
}  // namespace

void Simulator::ParSimulate(Crystal C, Detector &Det, SimulationSettings SS, SimulationOutput &Out, Settings &Options)
{
    if (!Det.Checklist.PixelMap) throw std::runtime_error("Detector needs a PixelMap");
    const size_t npix = Det.Pixels();
    // pixel orientation and size from the pixel map, IAC/Simulator.cpp:1282-1333
    if (SS.AutoPixelOrientation || SS.AutoPixelSize) {
        double v[6];
        for (int d = 0; d < 3; d++) {
            v[d] = Det.PixelMap[d + 3] - Det.PixelMap[d];
            v[3 + d] = Det.PixelMap[d + 3 * Det.DetectorSize[1]] - Det.PixelMap[d];
        }
        const double n0 = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double n1 = std::sqrt(v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
        if (SS.AutoPixelSize) {
            SS.PixelSize[0] = n0;
            SS.PixelSize[1] = n1;
        }
        if (SS.AutoPixelOrientation)
            for (int d = 0; d < 3; d++) {
                SS.PixelOrientationVectors[d] = v[d] / n0;
                SS.PixelOrientationVectors[3 + d] = v[3 + d] / n1;
            }
    }
    // sub-pixel steps, IAC/Simulator.cpp:745-760
    iac_sim_params sp{};
    sp.subsampling = (int)SS.SubSampling;
    const double *pv = SS.PixelOrientationVectors;
    double t = 1.0 / std::sqrt(pv[0] * pv[0] + pv[1] * pv[1] + pv[2] * pv[2]);
    t = (t / ((double)(2 * SS.SubSampling + 1))) * SS.PixelSize[0];
    for (int d = 0; d < 3; d++) sp.u_step[d] = pv[d] * t;
    t = 1.0 / std::sqrt(pv[3] * pv[3] + pv[4] * pv[4] + pv[5] * pv[5]);
    t = (t / ((double)(2 * SS.SubSampling + 1))) * SS.PixelSize[1];
    for (int d = 0; d < 3; d++) sp.v_step[d] = pv[3 + d] * t;
    sp.wavelength = SS.Wavelength;
    sp.intensity_squared = SS.IntensitySquared ? 1 : 0;
    sp.accurate_sincos = 0;

    iac_crystal_params cp{};
    cp.incoherent = SS.CrystSettings.Incoherent;
    cp.fluorescence_yield = SS.CrystSettings.FlYield;
    cp.random_orientation = SS.CrystSettings.RandOrientation;
    cp.isotropy = SS.CrystSettings.Isotropie;
    iac_photon_params pp{};
    pp.expected_photons = (double)SS.AveragePhotonesPerEmitterOnDetector * (double)SS.CrystSettings.FlYield *
                          (double)C.AtomPositions.size();
    pp.poisson = SS.PoissonSample;
    pp.adu_noise = SS.ADUNoise;
    pp.value_per_photon = SS.Value_per_Photon;
    uint64_t seed = SS.Seed;
    if (!seed) {
        std::random_device rd;
        seed = ((uint64_t)rd() << 32) ^ rd();
    }

    iac_ctx *ctx = Options.Context();
    void *s = Options.Stream();
    const uint32_t na = (uint32_t)C.AtomPositions.size(), nm = SS.Modes;
    const uint32_t chunk = std::max(1u, std::min(SS.FramesPerLaunch, SS.NumberOfSimulations));
    std::vector<double> atoms(3 * (size_t)na);
    for (size_t i = 0; i < na; i++)
        for (int d = 0; d < 3; d++) atoms[3 * i + d] = C.AtomPositions[i][d];
    DevBuf dA(ctx, atoms.size() * 8), dPM(ctx, npix * 12), dEm(ctx, (size_t)chunk * nm * na * 16),
        dCnt(ctx, (size_t)chunk * nm * 4), dRot(ctx, (size_t)chunk * 36), dI(ctx, (size_t)chunk * npix * 4);
    Check(iac_memcpy_h2d(ctx, dA.p, atoms.data(), atoms.size() * 8, s), "copy atoms");
    Check(iac_memcpy_h2d(ctx, dPM.p, Det.PixelMap, npix * 12, s), "copy pixel map");

    Out.Intensities.clear();
    Out.HitEvents.clear();
    Out.DetectorSize[0] = Det.DetectorSize[0];
    Out.DetectorSize[1] = Det.DetectorSize[1];
    std::vector<float> img((size_t)chunk * npix), rot((size_t)chunk * 9);
    for (uint32_t f0 = 0; f0 < SS.NumberOfSimulations; f0 += chunk) {
        const uint32_t nf = std::min(chunk, SS.NumberOfSimulations - f0);
        // frames f0.. use streams f0.. of the seed (emitters keyed per launch offset)
        Check(iac_crystal_emitters(ctx, (const double *)dA.p, na, nf, nm, &cp, seed + f0, (float *)dEm.p,
                                   (uint32_t *)dCnt.p, (float *)dRot.p, nullptr, s),
              "iac_crystal_emitters");
        Check(iac_simulate_intensity(ctx, (const float *)dPM.p, npix, (const float *)dEm.p, (const uint32_t *)dCnt.p,
                                     na, nm, nf, &sp, (float *)dI.p, s),
              "iac_simulate_intensity");
        Check(iac_simulate_photons(ctx, (float *)dI.p, npix, nf, f0, &pp, seed, s), "iac_simulate_photons");
        Check(iac_memcpy_d2h(ctx, img.data(), dI.p, (size_t)nf * npix * 4, s), "copy frames");
        Check(iac_memcpy_d2h(ctx, rot.data(), dRot.p, (size_t)nf * 36, s), "copy rotations");
        Check(iac_stream_synchronize(ctx, s), "synchronize");
        for (uint32_t f = 0; f < nf; f++) {
            const float *I = &img[(size_t)f * npix];
            Out.Intensities.emplace_back(I, I + npix);
            Settings::HitEvent e;
            std::copy(&rot[9 * (size_t)f], &rot[9 * (size_t)f] + 9, e.RotMatrix);
            e.SerialNumber = (int)(f0 + f);
            e.Event = (int)(f0 + f);
            e.Filename = SS.Filename_Intensity;
            e.Dataset = SS.Dataset;
            // IAC/Simulator.cpp:911-918: float sum, photon count, mean
            float sum = 0.0f;
            for (size_t j = 0; j < npix; j++) sum += I[j];
            double mean = sum;
            e.PhotonCount = (int)std::floor((mean / ((double)SS.Value_per_Photon)) + 0.5);
            e.MeanIntensity = (float)(mean / (double)npix);
            Out.HitEvents.push_back(e);
        }
    }
    if (SS.SaveResults) SaveSimulationOutput(Out, SS.Filename_Intensity, SS.Filename_XML, SS, Options);
}

void Simulator::SaveSimulationOutput(SimulationOutput &Out, std::string FnI, std::string FnX, SimulationSettings,
                                     Settings &Options)
{
    std::FILE *f = std::fopen(FnI.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + FnI);
    for (auto &I : Out.Intensities)
        if (std::fwrite(I.data(), sizeof(float), I.size(), f) != I.size()) {
            std::fclose(f);
            throw std::runtime_error("short write to " + FnI);
        }
    std::fclose(f);
    for (auto &e : Out.HitEvents) e.Filename = FnI;
    Options.SafeHitEventListToFile(FnX, Out.HitEvents);
}

void Simulator::GeneratePixelMap(int SizeA, int SizeB, float PixelSize, std::array<float, 3> Center,
                                 std::array<float, 3> VecA, std::array<float, 3> VecB, std::vector<float> &PM)
{
    float na = std::sqrt(VecA[0] * VecA[0] + VecA[1] * VecA[1] + VecA[2] * VecA[2]);
    float nb = std::sqrt(VecB[0] * VecB[0] + VecB[1] * VecB[1] + VecB[2] * VecB[2]);
    for (int d = 0; d < 3; d++) {
        VecA[d] = VecA[d] / na;
        VecB[d] = VecB[d] / nb;
    }
    PM.assign(3 * (size_t)SizeA * SizeB, 0.0f);
    for (int a = 0; a < SizeA; a++)
        for (int b = 0; b < SizeB; b++)
            for (int d = 0; d < 3; d++)
                PM[3 * (size_t)a * SizeB + 3 * (size_t)b + d] =
                    (float)(Center[d] + VecA[d] * PixelSize * (a - 0.5 * SizeA) + VecB[d] * PixelSize * (b - 0.5 * SizeB));
}

}  // namespace iac
