"""The autotuner's launch-parameter table (include/b200enc.h, B200ENC_TUNE_*)
on the CPU: it is host state only, so the library loads and answers without
a GPU. Names, ranges, the "name value" file the C callers load, and the
Python side's file writer agree."""
import subprocess
import sys
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(code, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=e, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout.strip()


PRE = ("import sys; sys.path.insert(0, 'bc250-vaapi_b200'); import b200enc; from b200enc import autotune; "
       "L = b200enc.load_library(); ")


def test_names_match_the_python_keys():
    out = _run(PRE + "print(','.join(L.b200enc_tune_name(k).decode() for k in range(8)), L.b200enc_tune_name(8))")
    names, last = out.split()
    assert last == "None"
    sys.path.insert(0, os.path.join(ROOT, "bc250-vaapi_b200"))
    from b200enc import autotune
    assert {n: i for i, n in enumerate(names.split(","))} == autotune.KEYS


def test_set_get_ranges():
    out = _run(PRE + "print(L.b200enc_tune_get(0), L.b200enc_tune_set(0, 3), L.b200enc_tune_get(0), "
               "L.b200enc_tune_set(0, 7), L.b200enc_tune_set(1, 3), L.b200enc_tune_set(1, 4), "
               "L.b200enc_tune_set(2, 17), L.b200enc_tune_set(4, 68), L.b200enc_tune_set(9, 1), "
               "L.b200enc_tune_get(9), L.b200enc_tune_set(0, 0), L.b200enc_tune_get(0), "
               "L.b200enc_tune_set(5, 3), L.b200enc_tune_set(5, 1))")
    assert out.split() == ["0", "0", "3", "-1", "-1", "0", "-1", "0", "-1", "-1", "0", "0", "-1", "0"]


def test_tune_file_round_trip(tmp_path):
    p = tmp_path / "tune.txt"
    _run(PRE + f"autotune.write_tune_file({str(p)!r}, {{'deblock_rows': 5, 'pchain_mbs_per_cta': 2, "
               "'rescore_ctas_per_sm': 12, 'fallback_ctas_per_sm': 4, 'intra_ctas': 34, 'me_stage': 1})")
    text = p.read_text()
    assert "deblock_rows 5" in text and text.startswith("#")
    # loaded explicitly
    out = _run(PRE + f"print(L.b200enc_tune_load({str(p)!r}.encode()), [L.b200enc_tune_get(k) for k in range(6)])")
    assert out == "6 [5, 2, 12, 4, 34, 1]"
    # loaded from the environment before the first use
    out = _run(PRE + "print([L.b200enc_tune_get(k) for k in range(6)])", env={"B200ENC_TUNE_FILE": str(p)})
    assert out == "[5, 2, 12, 4, 34, 1]"
    # out-of-range lines are skipped, the rest kept
    p.write_text("deblock_rows 9\npchain_mbs_per_cta 4\nbogus 3\n")
    out = _run(PRE + f"print(L.b200enc_tune_load({str(p)!r}.encode()), [L.b200enc_tune_get(k) for k in range(6)])")
    assert out == "1 [0, 4, 0, 0, 0, 0]"
    assert _run(PRE + "print(L.b200enc_tune_load(b'/nonexistent/tune.txt'))") == "-1"
