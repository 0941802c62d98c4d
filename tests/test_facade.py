"""The C++ classes with the reference's names (Settings, Detector, ACMesh,
AC1D, Simulator, RunIAC) and the iac_run driver: host-only checks here, and on
the GPU the reference's 3D and angular-averaged evaluations end to end from
files (pixel map, frame stack, XML event list) against the oracle."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "incohautocorrelate_b200")
RUN = os.path.join(PKG, "iac_run")


def _build_host_test():
    src = os.path.join(ROOT, "tests", "cpp", "test_facade_cpu.cpp")
    exe = os.path.join(ROOT, "tests", "cpp", "test_facade_cpu")
    if not os.path.exists(exe) or os.path.getmtime(exe) < os.path.getmtime(src) or \
            os.path.getmtime(exe) < os.path.getmtime(os.path.join(PKG, "libiac_facade.so")):
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
                        "-I", os.path.join(PKG, "cpp"), src, "-o", exe, "-L", PKG, "-liac_facade",
                        "-liac_b200", f"-Wl,-rpath,{PKG}"], check=True)
    return exe


def test_facade_host_checks(tmp_path):
    exe = _build_host_test()
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr + r.stdout


def _write_events(path, rots, mean_int, stack, counts):
    lines = ['<?xml version="1.0" encoding="utf-8"?>', "<root><Info><Size>%d</Size><Version>9</Version></Info><Content>" % len(rots)]
    for i, R in enumerate(rots):
        rot = "; ".join("%f" % float(v) for v in R)
        lines.append(f"<N{i}><Filename>{stack}</Filename><Dataset>data</Dataset><Event>{i}</Event>"
                     f"<SerialNumber>{i}</SerialNumber><MeanIntensity>{mean_int[i]}</MeanIntensity>"
                     f"<PhotonCount>{counts[i]}</PhotonCount><SupplementInfo></SupplementInfo>"
                     f"<Rotation>{rot}</Rotation></N{i}>")
    lines.append("</Content></root>")
    open(path, "w").write("".join(lines))


def _eval_xml(path, d, mesh, angular, step=1.0):
    open(path, "w").write(f"""<root><EvalSettings>
<InputFiles><EventList_Path>{d}/events.xml</EventList_Path><PixelMap_Path>{d}/pm.raw</PixelMap_Path>
<PixelMap_Dataset>40,56</PixelMap_Dataset><PixelMask_Path>{d}/mask.raw</PixelMask_Path></InputFiles>
<OutputFiles><AC_Final_Path>{d}/ac.bin</AC_Final_Path><AvIntensity_Path>{d}/avint.bin</AvIntensity_Path>
<Cq_Merged_Path>{d}/cq.bin</Cq_Merged_Path><Cq_small_Path>{d}/cqs.bin</Cq_small_Path>
<ACuw_Path>{d}/acuw.bin</ACuw_Path><Q_Vector>{d}/q.bin</Q_Vector></OutputFiles>
<OutputMesh><MeshSize>{mesh}</MeshSize><AngularAveraged>{str(angular).lower()}</AngularAveraged></OutputMesh>
<PhotonThreshold><PhotonOffset>0</PhotonOffset><PhotonStep>{step}</PhotonStep></PhotonThreshold>
<Misc><EchoLevel>0</EchoLevel></Misc></EvalSettings></root>""")


def _dataset(d, nframes=150, seed=4, rates=(0.08,)):
    """40x56 coarse flat detector, 5 % masked, frames of Poisson photon counts
    (mean rates[f % len(rates)] per pixel) scaled to ADU, random
    orientations; written as the raw files the driver reads."""
    from incohautocorrelate_b200 import workloads as W
    rng = np.random.default_rng(seed)
    ny, nx = 40, 56
    pm = W.flat_pixel_map(ny, nx, pitch=5e-4, dist=0.1)
    mask = W.random_mask(ny * nx, 0.05, seed)
    lam = np.array([rates[f % len(rates)] for f in range(nframes)])[:, None]
    frames = (rng.poisson(lam, (nframes, ny * nx)) * 1.0).astype(np.float32)
    rots = W.haar_rotations(nframes, seed + 1)
    rots = np.array([[float("%f" % v) for v in R] for R in rots], np.float32)  # as written to XML
    pm.tofile(f"{d}/pm.raw")
    mask.astype(np.int32).tofile(f"{d}/mask.raw")
    frames.tofile(f"{d}/stack.raw")
    _write_events(f"{d}/events.xml", rots, [-1.0] * nframes, f"{d}/stack.raw", [-1] * nframes)
    return pm, mask, frames, rots


def _averaged(frames, mask, step):
    """Detector::LoadAndAverageIntensity with photon discretisation
    (IAC/Detector.cpp:687-790): per-frame masked photon images, their sum
    rounded per pixel, times 1/N; MeanIntensity = photon sum / pixels."""
    n, npix = frames.shape
    disc = np.zeros(npix, np.int64)
    means = []
    for f in range(n):
        t = (frames[f] * mask.astype(np.float32)).astype(np.float32)
        ph = np.where(t >= 0, np.ceil((t - np.float32(0)) / np.float32(step)) * (t >= 0), 0).astype(np.float32)
        disc += np.floor(ph.astype(np.float64) + 0.5).astype(np.int64)
        s = np.float32(0)
        for v in ph:
            s = np.float32(s + v)
        means.append(np.float32(s / np.float32(npix)))
    I = disc.astype(np.float32) * np.float32(1.0 / np.float32(n))
    return (I * mask.astype(np.float32)).astype(np.float32), np.array(means, np.float32)


@pytest.mark.gpu
def test_iac_run_3d_evaluation_matches_oracle(tmp_path, oracle_lib):
    import ctypes as C
    o = oracle_lib
    d = str(tmp_path)
    pm, mask, frames, rots = _dataset(d)
    _eval_xml(f"{d}/eval.xml", d, 31, False)
    r = subprocess.run([RUN, "-e", f"{d}/eval.xml"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    km, mq = o.calc_kmap(pm)
    npix = km.size // 3
    # averaged intensity and event weights
    I, means = _averaged(frames, mask, 1.0)
    # sparse pairs: reference route choice per frame, photon lists of masked frames
    shape = o.big_mesh_shape(mq, 31)
    hl, off = [], [0]
    for f in range(len(frames)):
        t = (frames[f] * mask.astype(np.float32)).astype(np.float32)
        out = np.zeros((npix, 4), np.float32)
        n = o.lib().iaco_sparse_hitlist(o.p(t), o.p(km), npix, 0.0, 1.0, 1, o.p(out))
        hl.append(out[:n])
        off.append(off[-1] + n)
    ph = np.concatenate(hl)
    mesh, _ = o.sparse_batch(ph, np.array(off, np.uint64), rots, shape, cpu_gpu=-1, det_pixels=npix)
    acuw = np.fromfile(f"{d}/acuw.bin", np.float64)
    want_acuw = (mesh.astype(np.float32) * np.float32(0.001)).astype(np.float64)
    np.testing.assert_array_equal(acuw, want_acuw)
    # small C(q) of the averaged intensity
    Iav = np.fromfile(f"{d}/avint.bin", np.float32)
    Iav = (Iav * mask.astype(np.float32)).astype(np.float32)
    np.testing.assert_array_equal(Iav, I)
    s = o.small_cq_mesh_shape(mq, 31)
    mult = o.lib().iaco_cq_small_multiplicator(o.p(Iav), npix)
    small_u = np.zeros(s.size_ab * s.size_ab * s.size_c, np.uint64)
    o.lib().iaco_cq_small(o.p(Iav), o.p(km), npix, s, 0, mult, 0, npix, o.p(small_u))
    small = small_u.astype(np.float64) / mult
    np.testing.assert_array_equal(np.fromfile(f"{d}/cqs.bin", np.float64), small)
    # merged C(q) with MeanIntensity^2 weights
    nf = len(frames)
    rw = np.zeros(10 * nf, np.float32)
    mm = C.c_double()
    o.lib().iaco_cq_merge_weights(o.p(rots), o.p(means), nf, o.p(small), small.size, o.p(rw), C.byref(mm))
    big = np.zeros(s.size_ab ** 3, np.uint64)
    o.lib().iaco_cq_merge(o.p(small), o.p(rw), nf, s, 0, mm.value, 0, small.size, o.p(big))
    cq = big.astype(np.float64) / mm.value
    np.testing.assert_array_equal(np.fromfile(f"{d}/cq.bin", np.float64), cq)
    # final AC = AC_uw / C(q), 0 where C(q) <= 0
    final = np.zeros_like(cq)
    o.lib().iaco_merge_ac_and_cq(o.p(mesh), o.p(cq), cq.size, 0.001, 0.0, o.p(final))
    np.testing.assert_array_equal(np.fromfile(f"{d}/ac.bin", np.float64), final)


@pytest.mark.gpu
def test_iac_run_angular_averaged_evaluation_matches_oracle(tmp_path, oracle_lib):
    """Frames alternate between ~8 % and ~0.4 % hit pixels, so AC1D's sparse
    AC_UW takes both of the reference's routes (host loop below 0.75 %,
    IAC/AC1D.cpp:251-253); linear binning sums fractional floats, equal up to
    the order of the double additions."""
    o = oracle_lib
    d = str(tmp_path)
    pm, mask, frames, rots = _dataset(d, nframes=80, seed=9, rates=(0.08, 0.004))
    _eval_xml(f"{d}/eval.xml", d, 101, True)
    r = subprocess.run([RUN, "-e", f"{d}/eval.xml"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    km, mq = o.calc_kmap(pm)
    npix = km.size // 3
    I, _ = _averaged(frames, mask, 1.0)
    sh = o.ac1d_shape(mq, 101)
    mult = o.lib().iaco_ac1d_cq_multiplicator(o.p(I), npix)
    h = np.zeros(sh.size, np.uint64)
    o.lib().iaco_ac1d_cq(o.p(I), o.p(km), npix, sh, 1, mult, 0, npix, o.p(h))
    np.testing.assert_allclose(np.fromfile(f"{d}/cq.bin", np.float64), h.astype(np.float64) / mult,
                               rtol=1e-12, atol=0)
    hl, off = [], [0]
    for f in range(len(frames)):
        t = (frames[f] * mask.astype(np.float32)).astype(np.float32)
        out = np.zeros((npix, 4), np.float32)
        n = o.lib().iaco_sparse_hitlist(o.p(t), o.p(km), npix, 0.0, 1.0, 1, o.p(out))
        hl.append(out[:n])
        off.append(off[-1] + n)
    off = np.array(off, np.uint64)
    host = (np.diff(off).astype(np.float32) / np.float32(npix)) < np.float32(0.0075)
    assert host.any() and not host.all()
    acuw = np.zeros(sh.size)
    o.lib().iaco_ac1d_uw_frames(o.p(np.ascontiguousarray(np.concatenate(hl))), o.p(off), len(frames), npix,
                                sh.max_q, sh.dq_per_step, sh.size, 1, -1, o.p(acuw))
    np.testing.assert_allclose(np.fromfile(f"{d}/acuw.bin", np.float64), acuw, rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_iac_run_simulation_writes_frames_and_events(tmp_path):
    from incohautocorrelate_b200 import workloads as W
    d = str(tmp_path)
    pm = (W.flat_pixel_map(64, 64, pitch=1e-3, dist=0.1) * np.float32(1e10)).astype(np.float32)
    pm.tofile(f"{d}/pm.raw")
    open(f"{d}/sim.xml", "w").write(f"""<root><Simulation>
<OutputPath_EventList>{d}/sim_events.xml</OutputPath_EventList><OutputPath_Intensities>{d}/sim.raw</OutputPath_Intensities>
<Wavelength>1.55</Wavelength><NumberOfPattern>37</NumberOfPattern><NumberOfModes>2</NumberOfModes>
<RandomOriented>true</RandomOriented><AveragePhotonesPerEmitterOnDetector>2.0</AveragePhotonesPerEmitterOnDetector>
<SubSampling>0</SubSampling><UnitCells>3; 3; 4</UnitCells><LatticeVector_1>4.0; 0.0; 0.0</LatticeVector_1>
<LatticeVector_2>0.0; 4.0; 0.0</LatticeVector_2><LatticeVector_3>0.0; 0.0; 4.0</LatticeVector_3>
<UnitCell><NumberOfEmittersPerUnitcell>1</NumberOfEmittersPerUnitcell><Emitter_1>0.0; 0.0; 0.0</Emitter_1></UnitCell>
<Seed>77</Seed><PixelMap_Path>{d}/pm.raw</PixelMap_Path><PixelMap_Dataset>64,64</PixelMap_Dataset>
</Simulation></root>""")
    r = subprocess.run([RUN, "-s", f"{d}/sim.xml"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    frames = np.fromfile(f"{d}/sim.raw", np.float32).reshape(37, 64 * 64)
    assert (frames == np.round(frames)).all() and frames.min() >= 0
    # 36 emitters x 2 photons expected per frame
    assert abs(frames.sum(axis=1).mean() - 72) < 10
    txt = open(f"{d}/sim_events.xml").read()
    assert "<Size>37</Size>" in txt and txt.count("<Rotation>") == 37
