"""Host-side helpers that need no GPU: the decaying-magnitude synthetic systems,
the traffic figures bench.py reads from the committed ncu summaries, its
clock-sample summary, and the batch command line's argument parsing."""
import importlib.util
import pathlib

import numpy as np
import pytest

from libcc_b200 import synthetic as S

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_with_decay_scales_each_virtual_index():
    no, nu, f = 3, 10, 0.75
    inp = S.generate(no, nu, 1)
    d = S.with_decay(inp, f)
    g = 2.0 ** (-f * np.arange(nu))
    # T2(a,b,i,j) at a + nu*(b + nu*(i + no*j)); VM(l,c,x,y) at l + no*(c + nu*(x + no*y))
    for a, b, i, j in [(0, 0, 0, 0), (3, 5, 1, 2), (9, 2, 2, 0)]:
        idx = a + nu * (b + nu * (i + no * j))
        assert np.isclose(d.t2[idx], inp.t2[idx] * g[a] * g[b], rtol=1e-15, atol=0)
        assert np.isclose(d.voe[idx], inp.voe[idx] * g[a] * g[b], rtol=1e-15, atol=0)
    for l, c, x, y in [(0, 4, 1, 2), (2, 9, 0, 0)]:
        idx = l + no * (c + nu * (x + no * y))
        assert np.isclose(d.vm[idx], inp.vm[idx] * g[c], rtol=1e-15, atol=0)
    ntr = nu * (nu + 1) // 2
    for x, r1, I, J in [(2, 4, 7, 3), (0, 0, 0, 0), (1, 9, 9, 9)]:
        k = (x * nu + r1) * ntr + I * (I + 1) // 2 + J
        assert np.isclose(d.vvvo[k], inp.vvvo[k] * g[r1] * g[I] * g[J], rtol=1e-15, atol=0)
    assert np.array_equal(d.eh, inp.eh) and np.array_equal(d.ep, inp.ep)
    z = S.with_decay(inp, 0.0)
    for name in ("t1", "t2", "vm", "voe", "vvvo"):
        assert np.array_equal(getattr(z, name), getattr(inp, name)), name


def test_bench_reads_traffic_from_the_committed_summaries():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    for kind in ("f64", "emu"):
        t = bench.read_traffic("no24-nu320", kind)
        assert t is not None and 1e9 < t < 5e9, (kind, t)
    assert bench.read_traffic("no-such-workload", "f64") is None


def test_clock_summary_reads_loaded_samples_and_reasons(tmp_path, monkeypatch):
    """The bench's clock evidence: median SM clock over the samples under load
    (power at least half the maximum), and every throttle reason seen active."""
    monkeypatch.setenv("CCT_CLOCKS_DIR", str(tmp_path))
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    cs = bench.ClockSampler(0)
    assert cs.path.parent == tmp_path
    rows = ["0, 1965, 1965, 150.0, 0x0, Not Active, Not Active, Not Active, Not Active",   # idle: ignored
            "0, 1750, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1730, 1965, 1001.0, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1760, 1965, 995.0, 0x0, Not Active, Not Active, Not Active, Not Active",
            "garbage line"]
    cs.path.write_text("\n".join(rows) + "\n")
    cs.proc = object()  # a sampler that ran
    s = cs.summary()
    assert s["sm_mhz"] == 1750.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3 and s["power_w_max"] == 1001.0
    cs.path.write_text("0, 1500, 1965, 900.0, 0x8, Not Active, Active, Not Active, Not Active\n")
    assert cs.summary()["reasons"] == ["hw_thermal_slowdown"]


def test_batch_command_line_parses_without_a_gpu(capsys):
    from libcc_b200 import batch
    with pytest.raises(SystemExit) as e:
        batch.main(["--help"])
    assert e.value.code == 0
    assert "--systems" in capsys.readouterr().out


def test_packed_vvvo_option_is_validated_without_a_gpu():
    """vvvo_mode out of range, or PACKED on an emulated plan, is rejected before any
    device call."""
    import ctypes
    from libcc_b200 import _native as N
    try:
        lib = N.load()
    except N.NativeLibraryError:
        pytest.skip("library not built")
    for prec, mode in ((N.CCT_PREC_FP64, 7), (N.CCT_PREC_INT8_EMU, N.CCT_VVVO_PACKED)):
        opt = N.Options()
        lib.ccT_options_default(ctypes.byref(opt))
        opt.precision, opt.vvvo_mode = prec, mode
        h = ctypes.c_void_p()
        assert lib.ccT_plan_create(ctypes.byref(h), 4, 10, ctypes.byref(opt)) == 1
