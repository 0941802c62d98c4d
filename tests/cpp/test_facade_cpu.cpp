// Host-only checks of the C++ classes with the reference's names: the XML
// property tree, the event-list file formats (IAC/Settings.cpp:473-676), the
// evaluation-settings loader (IAC/MainRunModes.cpp:32-91), FloatToInt and the
// crystal lattice (IAC/Crystal.cpp:192-229).  No device is touched.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>

#include "iac/RunIAC.h"
#include "iac/PropertyTree.h"

using namespace iac;

static int failures = 0;
#define EXPECT(c)                                                        \
    do {                                                                 \
        if (!(c)) {                                                      \
            std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #c); \
            failures++;                                                  \
        }                                                                \
    } while (0)

int main(int argc, char **argv)
{
    const std::string dir = argc > 1 ? argv[1] : ".";
    // property tree round trip with entities and nesting
    PropertyTree pt;
    pt.Put("root.A.B", "x<y & z");
    pt.Put("root.A.C", 42);
    pt.Put("root.D", 1.5);
    const PropertyTree back = PropertyTree::ParseXml(pt.ToXml());
    EXPECT(back.Get("root.A.B", std::string()) == "x<y & z");
    EXPECT(back.Get<int>("root.A.C", 0) == 42);
    EXPECT(back.Get<double>("root.D", 0.0) == 1.5);
    EXPECT(back.Get<int>("root.Missing", 7) == 7);

    // event list, version 9 (Rotation string) round trip
    Settings S;
    S.HitEvents.resize(3);
    for (int i = 0; i < 3; i++) {
        auto &e = S.HitEvents[i];
        const float R[9] = {0.5f, -0.25f, 0.125f, 1, 0, 0, 0, 0.75f, -1};
        for (int k = 0; k < 9; k++) e.RotMatrix[k] = R[k] * (i + 1);
        e.Filename = "stack.raw";
        e.Dataset = "data";
        e.Event = 10 + i;
        e.SerialNumber = i;
        e.MeanIntensity = 0.0625f * i;
        e.PhotonCount = 100 * i;
    }
    const std::string xml = dir + "/events.xml";
    S.SafeHitEventListToFile(xml);
    Settings L;
    L.LoadHitEventListFromFile(xml);
    EXPECT(L.HitEvents.size() == 3);
    for (int i = 0; i < 3; i++) {
        EXPECT(L.HitEvents[i].Event == 10 + i);
        EXPECT(L.HitEvents[i].PhotonCount == 100 * i);
        EXPECT(L.HitEvents[i].Filename == "stack.raw");
        for (int k = 0; k < 9; k++) EXPECT(std::fabs(L.HitEvents[i].RotMatrix[k] - S.HitEvents[i].RotMatrix[k]) < 1e-6);
    }
    // version 1 files keep R0..R8 under root.content.N<i>
    {
        std::ofstream f(dir + "/events_v1.xml");
        f << "<?xml version=\"1.0\"?><root><Info><Size>1</Size><Version>1</Version></Info><content><N0>"
             "<Filename>a</Filename><Dataset>d</Dataset><Event>5</Event><SerialNumber>0</SerialNumber>"
             "<MeanIntensity>0.5</MeanIntensity><PhotonCount>3</PhotonCount><R0>0</R0><R1>1</R1><R3>-1</R3>"
             "<R4>0</R4></N0></content></root>";
    }
    Settings V1;
    V1.LoadHitEventListFromFile(dir + "/events_v1.xml");
    EXPECT(V1.HitEvents.size() == 1 && V1.HitEvents[0].Event == 5);
    EXPECT(V1.HitEvents[0].RotMatrix[1] == 1 && V1.HitEvents[0].RotMatrix[3] == -1 && V1.HitEvents[0].RotMatrix[8] == 1);
    // inversion of a rotation is its transpose
    V1.InvertRotationMatrices();
    EXPECT(std::fabs(V1.HitEvents[0].RotMatrix[1] + 1) < 1e-7 && std::fabs(V1.HitEvents[0].RotMatrix[3] - 1) < 1e-7);

    // evaluation settings keys
    {
        std::ofstream f(dir + "/eval.xml");
        f << "<root><EvalSettings><InputFiles><EventList_Path>ev.xml</EventList_Path>"
             "<PixelMap_Path>pm.raw</PixelMap_Path><PixelMap_Dataset>4,6</PixelMap_Dataset></InputFiles>"
             "<OutputMesh><MeshSize>63</MeshSize><QZoom>1.5</QZoom><AngularAveraged>true</AngularAveraged>"
             "<AC_SecondMap_Flags><InterpolationMode>1</InterpolationMode></AC_SecondMap_Flags></OutputMesh>"
             "<PhotonThreshold><PhotonStep>2.5</PhotonStep></PhotonThreshold>"
             "<Misc><EchoLevel>0</EchoLevel></Misc></EvalSettings></root>";
    }
    Settings E;
    RunIAC::CreateDataEval_Settings ES = RunIAC::LoadEvaluationSettings(dir + "/eval.xml", E);
    EXPECT(ES.XML_Path == "ev.xml" && ES.PixelMap_DataSet == "4,6");
    EXPECT(ES.MeshSize == 63 && ES.QZoom == 1.5f && ES.AngularAveraged && ES.DoubleMap);
    EXPECT(ES.AC_FirstMap_Flags.InterpolationMode == Settings::NearestNeighbour);
    EXPECT(ES.AC_SecondMap_Flags.InterpolationMode == Settings::Linear);
    EXPECT(ES.PhotonStep == 2.5f && ES.PhotonOffset == 0.0f && !E.echo);

    // FloatToInt / IntToFloat with Step 0.001f (IAC/Settings.h:162-187)
    EXPECT(S.FloatToInt(1.0f) == 1000 && S.FloatToInt(4.0) == 4000);
    EXPECT(S.FloatToInt(10526.0) == 10526000 && S.FloatToInt(10527.0) == 10526999);

    // lattice centred at the origin, unit cell added per cell
    double LV[3][3] = {{4, 0, 0}, {0, 4, 0}, {0, 0, 4}};
    unsigned int cells[3] = {5, 5, 8};
    Crystal C(LV, cells, {{0, 0, 0}, {1, 0.5, 0}});
    EXPECT(C.AtomPositions.size() == 400);
    double cx = 0, cz = 0;
    for (size_t i = 0; i < C.AtomPositions.size(); i += 2) {
        cx += C.AtomPositions[i][0];
        cz += C.AtomPositions[i][2];
    }
    EXPECT(std::fabs(cx) < 1e-9 && std::fabs(cz) < 1e-9);
    EXPECT(C.AtomPositions[1][0] - C.AtomPositions[0][0] == 1.0);

    if (failures) {
        std::fprintf(stderr, "%d failure(s)\n", failures);
        return 1;
    }
    std::printf("facade host checks passed\n");
    return 0;
}
