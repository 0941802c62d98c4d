// Settings.cpp -- device context, echo and the XML event list
// (IAC/Settings.cpp:311-676).
#include "Settings.h"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <stdexcept>

#include "PropertyTree.h"

namespace iac {

void Check(iac_status st, const char *what)
{
    if (st != IAC_OK) {
        const char *m = iac_last_error();
        throw std::runtime_error(std::string(what) + ": " + iac_status_string(st) +
                                 (m && *m ? std::string(" (") + m + ")" : std::string()));
    }
}

Settings::Settings() {}

Settings::~Settings()
{
    if (ctx_) {
        if (stream_) iac_stream_destroy(ctx_, stream_);
        iac_ctx_destroy(ctx_);
    }
}

void Settings::Echo(std::string output)
{
    if (echo) std::cout << output << std::endl;
}

void Settings::SetUp_OpenCL() { SetUp_Device(0); }

void Settings::SetUp_Device(int device)
{
    if (ctx_) return;
    Check(iac_ctx_create(device, &ctx_), "iac_ctx_create");
    Check(iac_stream_create(ctx_, &stream_), "iac_stream_create");
    device_ = device;
}

iac_ctx *Settings::Context()
{
    if (!ctx_) SetUp_Device(0);
    return ctx_;
}

void *Settings::Stream()
{
    if (!ctx_) SetUp_Device(0);
    return stream_;
}

// ---------------------------------------------------------------------------
// event list, IAC/Settings.cpp:473-676
// ---------------------------------------------------------------------------
void Settings::SafeHitEventListToFile(std::string Filename) { SafeHitEventListToFile(Filename, HitEvents); }

void Settings::SafeHitEventListToFile(std::string Filename, std::vector<HitEvent> &List,
                                      bool AdditionalInformations,
                                      std::unordered_map<std::string, std::string> Info)
{
    PropertyTree pt;
    pt.Put("root.Info.Size", List.size());
    pt.Put("root.Info.Version", XML_HITLIST_VERSION);
    if (AdditionalInformations)
        for (auto &kv : Info) pt.Put("root.Info." + kv.first, kv.second);
    for (size_t i = 0; i < List.size(); i++) {
        const std::string p = "root.Content.N" + std::to_string(i);
        pt.Put(p + ".Filename", List[i].Filename);
        pt.Put(p + ".Dataset", List[i].Dataset);
        pt.Put(p + ".Event", List[i].Event);
        pt.Put(p + ".SerialNumber", List[i].SerialNumber);
        pt.Put(p + ".MeanIntensity", List[i].MeanIntensity);
        pt.Put(p + ".PhotonCount", List[i].PhotonCount);
        pt.Put(p + ".SupplementInfo", List[i].SupplementInfo);
        // the reference writes the matrix with std::to_string (six decimals)
        std::string rm = std::to_string(List[i].RotMatrix[0]);
        for (int j = 1; j < 9; j++) rm += "; " + std::to_string(List[i].RotMatrix[j]);
        pt.Put(p + ".Rotation", rm);
    }
    pt.WriteXml(Filename);
}

void Settings::LoadHitEventListFromFile(std::string Filename)
{
    const PropertyTree pt = PropertyTree::ReadXml(Filename);
    const unsigned int Size = pt.Get<unsigned int>("root.Info.Size", 0u);
    const unsigned int Version = pt.Get<unsigned int>("root.Info.Version", 1u);
    if (Size == 0) return;
    HitEvents.clear();
    std::string base;
    if (!pt.Find("root.content.N0.Filename") && !pt.Find("root.Content.N0.Filename"))
        base = "root.content.";
    else
        base = Version >= 2 ? "root.Content.N" : "root.content.N";
    for (unsigned int i = 0; i < Size; i++) {
        const std::string p = base + std::to_string(i);
        if (!pt.Find(p)) throw std::runtime_error("event list " + Filename + " lacks entry " + p);
        HitEvent t;
        t.Filename = pt.Get(p + ".Filename", std::string());
        t.Dataset = pt.Get(p + ".Dataset", std::string());
        t.Event = pt.Get<int>(p + ".Event", 0);
        t.SerialNumber = pt.Get<int>(p + ".SerialNumber", 0);
        t.MeanIntensity = pt.Get<float>(p + ".MeanIntensity", -1.0f);
        t.PhotonCount = pt.Get<int>(p + ".PhotonCount", -1);
        t.SupplementInfo = pt.Get(p + ".SupplementInfo", std::string());
        const float id[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        if (Version == 1) {
            for (int k = 0; k < 9; k++) t.RotMatrix[k] = pt.Get<float>(p + ".R" + std::to_string(k), id[k]);
        } else {
            std::string in = pt.Get(p + ".Rotation", std::string("1.0; 0.0; 0.0; 0.0; 1.0; 0.0; 0.0; 0.0; 1.0"));
            float v[9];
            int count = 0;
            bool ok = true;
            size_t pos;
            while ((pos = in.find(';')) != std::string::npos) {
                if (count >= 8) {
                    ok = false;
                    break;
                }
                v[count++] = (float)std::atof(in.substr(0, pos).c_str());
                in.erase(0, pos + 1);
            }
            if (ok && count == 8) {
                v[8] = (float)std::atof(in.c_str());
                for (int k = 0; k < 9; k++) t.RotMatrix[k] = v[k];
            } else {
                for (int k = 0; k < 9; k++) t.RotMatrix[k] = id[k];
            }
        }
        HitEvents.push_back(t);
    }
}

// inverse in double (the reference inverts with Eigen, IAC/Settings.cpp:535-556)
void Settings::InvertRotationMatrices()
{
    for (auto &e : HitEvents) {
        const double a = e.RotMatrix[0], b = e.RotMatrix[1], c = e.RotMatrix[2], d = e.RotMatrix[3],
                     f = e.RotMatrix[4], g = e.RotMatrix[5], h = e.RotMatrix[6], k = e.RotMatrix[7],
                     l = e.RotMatrix[8];
        const double A = f * l - g * k, B = -(d * l - g * h), C = d * k - f * h;
        const double det = a * A + b * B + c * C;
        const double inv[9] = {A / det, -(b * l - c * k) / det, (b * g - c * f) / det,
                               B / det, (a * l - c * h) / det,  -(a * g - c * d) / det,
                               C / det, -(a * k - b * h) / det, (a * f - b * d) / det};
        for (int m = 0; m < 9; m++) e.RotMatrix[m] = (float)inv[m];
    }
}

// ---------------------------------------------------------------------------
// frame sources
// ---------------------------------------------------------------------------
void RawStackSource::Load(const std::string &filename, const std::string &, int event, float *intensity,
                          size_t npix)
{
    std::FILE *f = std::fopen(filename.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open frame stack " + filename);
    if (std::fseek(f, (long)((size_t)event * npix * sizeof(float)), SEEK_SET) != 0 ||
        std::fread(intensity, sizeof(float), npix, f) != npix) {
        std::fclose(f);
        throw std::runtime_error("frame " + std::to_string(event) + " missing in " + filename);
    }
    std::fclose(f);
}

void MemoryFrameSource::Load(const std::string &, const std::string &, int event, float *intensity,
                             size_t npix)
{
    if (event < 0 || (size_t)event >= Frames.size() || Frames[event].size() != npix)
        throw std::runtime_error("frame " + std::to_string(event) + " not in memory");
    std::copy(Frames[event].begin(), Frames[event].end(), intensity);
}

}  // namespace iac
