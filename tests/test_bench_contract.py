"""The bench's check of calibration results against the reference's numerical contract
(bench.calibration_contract, restating tests/numerics/support.h:45-57,119-142,181-226): the
contract rows' expected words pass, wrong words are caught, and the host two-rounding form
passes on every combination of the special words those rows use (the reference asserts the
same of its host form, tests/numerics_test.cpp:79-100)."""
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(HERE, "..", "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def rows():
    with open(os.path.join(HERE, "golden", "calibration_contract_rows.json")) as f:
        return json.load(f)


def words(key, sel):
    return np.array([int(r[key], 16) for r in sel], np.uint32).view(np.float32)


def test_contract_rows_pass_and_wrong_words_fail():
    b, sel = bench(), rows()
    x, o, g, want = (words(k, sel) for k in ("x", "offset", "gain", "expected"))
    report = b.calibration_contract(x, o, g, want)
    assert report["violations"] == 0, report
    assert sum(report["classes"].values()) == len(sel)
    assert all(report["classes"][k] > 0 for k in ("nan_input", "invalid", "infinite", "overflow",
                                                  "zero", "subnormal", "normal"))
    notes = [r["note"] for r in sel]
    wrong = want.copy().view(np.uint32)
    wrong[notes.index("(1 + 2^-23 - 1) * 1e8 is exact")] += 2        # 2 ulp off
    wrong[notes.index("(5 - 5) * -3 is -0")] = 0x00000000           # zero of the wrong sign
    wrong[notes.index("NaN gain")] = 0x3f800000                      # NaN input, finite result
    # A subnormal result may be off by one unit of 2^-149, as the reference's check allows (a
    # flushed 2^-149 passes it, and only the row's exact word catches that); two units fail.
    wrong[notes.index("2^-149 is not flushed")] = 0x00000003
    assert b.calibration_contract(x, o, g, wrong.view(np.float32))["violations"] == 4


def test_host_form_meets_contract_on_special_words(oracle_lib):
    b, sel = bench(), rows()
    special = np.unique(np.concatenate([words(k, sel).view(np.uint32)
                                        for k in ("x", "offset", "gain")]))
    n = special.size
    idx = np.arange(n ** 3)
    x = special[idx % n].reshape(n * n, n)
    o = special[idx // n % n].view(np.float32).reshape(n * n, n)
    g = special[idx // n // n].view(np.float32).reshape(n * n, n)
    host = oracle_lib.calibrate_image(x, o, g)
    report = b.calibration_contract(x.view(np.float32), o, g, host)
    assert report["violations"] == 0, report
    assert report["max_ulp_normal"] <= 1.5
