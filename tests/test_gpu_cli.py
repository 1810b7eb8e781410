"""The settings-file runner (digHoloRunBatchFromConfigFile, digHolo.h:1962,
digHolo.cpp:16766-17931) and its command-line program digholo_run.

A settings file asking for simulated frames (FrameBufferFilename with no
value: 15 frames of 320 x 256 pixels, one polarisation, 5 mode groups,
frame f exciting mode f), AutoAlign of tilt, centre and waist, and every
output file.  Run through the library call, through digholo_run and, where
present, through the reference build's own runner in its own directory:
the output files exist with the sizes the summary implies, each frame's
largest coefficient sits at its own mode, the summary lists the same keys as
the reference's, and IL agrees with the reference's within 0.05 dB.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import ref_lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SETTINGS = """FrameBufferFilename
FrameWidth\t320
FrameHeight\t256
BatchCount\t15
PolCount\t1
PixelSize\t20e-6
WavelengthCentre\t1565e-9
fftWindowSizeX\t256
fftWindowSizeY\t256
IFFTResolutionMode\t1
MaxMG\t5
AutoAlignTilt\t1
AutoAlignCentre\t1
AutoAlignWaist\t1
AutoAlignDefocus\t0
OutputFilenameSummary\tsummary.txt
OutputFilenameCoefs\tcoefs.bin
OutputFilenameFields\tfields.bin
OutputFilenameBasis\tbasis.bin
OutputFilenameXaxis\tx.bin
OutputFilenameYaxis\ty.bin
"""


@pytest.fixture(scope="module")
def lib():
    import digholo_b200
    return digholo_b200.load()


def _summary(path):
    out = {}
    for line in open(path).read().replace("\r", "").splitlines():
        parts = line.split("\t")
        if len(parts) >= 2:
            out[parts[0]] = parts[1:]
    return out


def _check_outputs(d):
    s = _summary(os.path.join(d, "summary.txt"))
    w, h = int(s["FieldWidth"][0]), int(s["FieldHeight"][0])
    coefs = np.fromfile(os.path.join(d, "coefs.bin"), dtype=np.complex64).reshape(15, -1)
    assert coefs.shape[1] == 15
    fields = np.fromfile(os.path.join(d, "fields.bin"), dtype=np.complex64)
    assert fields.size == 15 * w * h
    assert np.fromfile(os.path.join(d, "basis.bin"), dtype=np.complex64).size == 15 * w * h
    assert np.fromfile(os.path.join(d, "x.bin"), dtype=np.float32).size == w
    assert np.fromfile(os.path.join(d, "y.bin"), dtype=np.float32).size == h
    assert os.path.getsize(os.path.join(d, "testFrame.bin")) == 15 * 320 * 256 * 2
    hits = int((np.abs(coefs).argmax(axis=1) == np.arange(15)).sum())
    assert hits >= 14, hits
    return s


def _run_python(d, module):
    """The runner called from a fresh Python process (it works on handle 0
    when one exists, as the reference's does), in directory d."""
    open(os.path.join(d, "settings.txt"), "w").write(SETTINGS)
    load = "import ref_lib; L = ref_lib.load()" if module == "ref" else "import digholo_b200; L = digholo_b200.load()"
    code = ("import sys; sys.path[:0] = [%r, %r]; %s; sys.exit(L.digHoloRunBatchFromConfigFile(b'settings.txt'))"
            % (os.path.join(ROOT, "oracle"), ROOT, load))
    r = subprocess.run([sys.executable, "-c", code], cwd=d, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def test_runner_call_and_program(lib, tmp_path):
    a = tmp_path / "call"
    a.mkdir()
    _run_python(str(a), "ours")
    sa = _check_outputs(str(a))
    b = tmp_path / "program"
    b.mkdir()
    open(b / "settings.txt", "w").write(SETTINGS)
    r = subprocess.run([os.path.join(ROOT, "digholo_b200", "digholo_run"), "settings.txt"], cwd=str(b),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    sb = _check_outputs(str(b))
    assert abs(float(sa["IL"][0]) - float(sb["IL"][0])) < 1e-3
    if ref_lib.available():
        # the reference's runner works on its handle 0: a fresh process
        c = tmp_path / "reference"
        c.mkdir()
        _run_python(str(c), "ref")
        sc = _summary(str(c / "summary.txt"))
        assert set(sa) == set(sc)
        print("IL: this build %s, reference %s" % (sa["IL"][0], sc["IL"][0]))
        assert abs(float(sa["IL"][0]) - float(sc["IL"][0])) <= 0.05
