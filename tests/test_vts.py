"""VTS output (reference: src/io/VTSwriter.cu) -- the oracle and the CUDA path against .vts
files written by the reference's own VTSwriter.

tests/golden/vts/<case>_t<step>.vts.gz were written by the reference's VTSwriter, run by
the -fmad=false reference build in main.cu's call sequence (make_golden.py --vts).  The
oracle's text restatement must reproduce them byte for byte from the reference's own
field dumps (CPU); the FP64 CUDA path, bit-exact with that build, must write the same
bytes (GPU).  The binary formats carry the values of clipb_get_fields exactly (Float64)
or rounded to Float32.
"""
import gzip
import os
import re

import numpy as np
import pytest

from conftest import golden_config, golden_npz
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
VTS = os.path.join(HERE, "golden", "vts")
# (case, step) pairs with a reference-written file
CASES = [("drop2d_small", 0), ("drop2d_small", 10), ("drop2d_small", 50), ("inlet2d_small", 0),
         ("inlet2d_small", 30), ("drop3d_small", 0), ("drop3d_small", 20)]


def reference_vts(name, step):
    with gzip.open(os.path.join(VTS, f"{name}_t{step}.vts.gz"), "rb") as fp:
        return fp.read()


@pytest.mark.parametrize("name,step", CASES)
def test_oracle_vts_text_equals_reference_writer(name, step):
    a = np.load(golden_npz(name + "_nofma"))
    dim = 3 if "3d" in name else 2
    text = O.vts_text(dim, a[f"c_{step}"], a[f"p_{step}"], a[f"rho_{step}"], a[f"vel_{step}"])
    assert text.encode() == reference_vts(name, step)


def test_reference_vts_fixture_shape():
    """The fixture is the reference's text layout: extents over the interior, four arrays."""
    t = reference_vts("drop2d_small", 10).decode()
    assert '<StructuredGrid WholeExtent="1 24 1 32 0 0">' in t
    assert re.findall(r'Name="(\w+)"', t) == ["Velocity", "C", "P", "Rho"]
    assert 'NumberOfComponents="2"' in t
    t3 = reference_vts("drop3d_small", 0).decode()
    assert '<StructuredGrid WholeExtent="1 16 1 20 1 14">' in t3


def parse_binary(path):
    """Arrays of an appended-raw .vts file written by clipb_write_vts (UInt64 headers)."""
    with open(path, "rb") as fp:
        raw = fp.read()
    mark = b'<AppendedData encoding="raw">\n_'
    head, body = raw.split(mark, 1)
    head = head.decode()
    assert 'header_type="UInt64"' in head
    decl = re.findall(r'<DataArray type="(Float\d\d)"([^>]*)offset="(\d+)"/>', head)
    out = {}
    for typ, attrs, off in decl:
        name = re.search(r'Name="(\w+)"', attrs)
        name = name.group(1) if name else "Points"
        ncomp = re.search(r'NumberOfComponents="(\d)"', attrs)
        ncomp = int(ncomp.group(1)) if ncomp else 1
        off = int(off)
        nbytes = int(np.frombuffer(body[off:off + 8], dtype="<u8")[0])
        dt = "<f8" if typ == "Float64" else "<f4"
        out[name] = np.frombuffer(body[off + 8:off + 8 + nbytes], dtype=dt).reshape(-1, ncomp)
    assert body.endswith(b"\n</AppendedData>\n</VTKFile>\n")
    return head, out


def interior_points(s, field):
    """Interior of a reference-layout field in VTS point order (x fastest), comp last."""
    a = s.interior_field(field)
    return a.transpose(2, 1, 0, 3).reshape(-1, a.shape[3])


@pytest.mark.gpu
@pytest.mark.parametrize("name,step", CASES)
def test_vts_ascii_equals_reference_writer(name, step, tmp_path):
    import clip_b200 as cb
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init()
        s.solve(step)
        path = s.write_vts(tmp_path, "results", "ascii")
        assert os.path.basename(path) == f"results_t{step}.vts"
        with open(path, "rb") as fp:
            mine = fp.read()
    ref = reference_vts(name, step)
    if mine != ref:
        a, b = mine.split(b"\n"), ref.split(b"\n")
        k = 0
        while k < min(len(a), len(b)) and a[k] == b[k]:
            k += 1
        pytest.fail(f"line {k}: {a[k] if k < len(a) else None!r} vs {b[k] if k < len(b) else None!r}")


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("name", ["drop2d_small", "drop3d_small"])
def test_vts_binary_carries_the_fields(name, prec, tmp_path):
    import clip_b200 as cb
    with cb.Solver(golden_config(name), prec) as s:
        s.init()
        s.solve(7)
        p64 = s.write_vts(tmp_path / "b64", "results", "binary64")
        p32 = s.write_vts(tmp_path / "b32", "results", "binary32")
        want = {"Velocity": interior_points(s, "vel"), "C": interior_points(s, "c"),
                "P": interior_points(s, "p"), "Rho": interior_points(s, "rho")}
        n = s.interior
    head, got = parse_binary(p64)
    ext = f"1 {n[0]} 1 {n[1]} " + (f"1 {n[2]}" if len(n) == 3 and "3d" in name else "0 0")
    assert f'WholeExtent="{ext}"' in head
    for k, v in want.items():
        np.testing.assert_array_equal(got[k], v, err_msg=k)
    _, got32 = parse_binary(p32)
    for k, v in want.items():
        np.testing.assert_array_equal(got32[k], v.astype(np.float32), err_msg=k)
    pts = got["Points"]
    assert pts.shape == (want["C"].shape[0], 3)
    assert pts[0].tolist() == [1, 1, 1 if "3d" in name else 0]
    assert pts[1].tolist() == [2, 1, 1 if "3d" in name else 0]
    assert pts[-1].tolist() == [n[0], n[1], n[2] if "3d" in name else 0]


@pytest.mark.gpu
def test_vts_async_writes_overlap_steps(tmp_path):
    """Writes queued while the solver keeps stepping hold the state of their own step."""
    import clip_b200 as cb
    cfg = golden_config("rti2d_small")
    with cb.Solver(cfg, "fp32") as a, cb.Solver(cfg, "fp32") as b:
        a.init()
        b.init()
        want = {}
        for k in range(6):
            a.solve(5)
            a.write_vts(tmp_path, "run", "binary64", wait=False)
            b.solve(5)
            want[b.steps] = {"C": interior_points(b, "c"), "Velocity": interior_points(b, "vel"),
                             "P": interior_points(b, "p")}
        a.vts_wait()
        for step, fields in want.items():
            _, got = parse_binary(tmp_path / f"run_t{step}.vts")
            for k, v in fields.items():
                np.testing.assert_array_equal(got[k], v, err_msg=f"{k} step {step}")


@pytest.mark.gpu
def test_vts_errors(tmp_path):
    import clip_b200 as cb
    blocker = tmp_path / "file"
    blocker.write_text("not a folder")
    with cb.Solver(golden_config("drop2d_small"), "fp32") as s:
        with pytest.raises(cb.ClipError):
            s.write_vts(tmp_path, "x", "ascii")  # before init
        s.init()
        with pytest.raises(cb.ClipError):
            s.write_vts(blocker, "x", "ascii")  # the folder cannot be created
        # the file cannot be opened: reported by the writer thread, raised by vts_wait
        s.write_vts(tmp_path, "missing_dir/x", "binary32", wait=False)
        with pytest.raises(cb.ClipError, match="missing_dir"):
            s.vts_wait()
        s.vts_wait()  # the error is reported once
        s.solve(2)
        s.write_vts(tmp_path, "ok", "binary32")
        assert (tmp_path / "ok_t2.vts").exists()


@pytest.mark.gpu
def test_vts_writer_mirror_follows_output_interval(tmp_path):
    """Reference-shaped loop of main.cu:78-86 with VTSwriter.writeToFile every step."""
    import clip_b200 as cb
    text = open(golden_config("drop2d_small")).read().replace("outputInterval = 1000", "outputInterval = 4")
    cfg = tmp_path / "config.txt"
    cfg.write_text(text)
    idata = cb.InputData(str(cfg), "fp64")
    dom = cb.Domain(idata)
    DA = cb.DataArray(idata, dom)
    ns = cb.NSAllen(idata, dom, DA)
    ti = cb.TimeInfo(idata, ns.solver)
    w = cb.VTSwriter(DA, idata, dom, ti, str(tmp_path / "results"), "results")
    ns.initialCondition()
    DA.updateDevice()
    ns.deviceInitializer()
    w.writeToFile()
    for _ in range(10):
        ns.solve()
        ti.increment()
        w.writeToFile()
    files = sorted(os.listdir(tmp_path / "results"))
    assert files == ["results_t0.vts", "results_t4.vts", "results_t8.vts"]
    assert ti.getFinalStep() == 1000
