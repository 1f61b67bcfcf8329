"""Host-side helpers of bench.py (no GPU): the name of the level-1 kernel the
launch-shape tuner chose, read from its report.

The tuner's level-1 keys end in the visit kind (y0: first visit, y1: with the
iterate, timed in its final-visit form) and carry the number of blocked
candidates (b2: the blocked kernel at 512 and 256 threads; b3: also its staged
form) after the natural kernel's thread counts.
"""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_level1_kernel_names_follow_the_tuner_table():
    b = _bench()
    tune = {
        "ic_apply|f32|n4096|c4096|l256|b3|y0|f": [1, [334.2, 271.4, 318.5, 285.7]],
        "ic_apply|f32|n4096|c4096|l256|b3|y1|f": [3, [578.9, 484.4, 428.4, 412.7, 642.4, 512.3, 761.9, 436.6]],
        "ic_apply|f64|n4096|c4096|l256|b3|y0|f": [3, [784.4, 591.0, 681.3, 507.6]],
        "ic_apply|f64|n4096|c4096|l256|b2|y1|f": [6, [1201.8, 964.0, 835.9, 770.7, 736.6, 1107.6, 1712.1]],
        "prolong|f32|n4096|c4096|k6": [0, [93.9, 94.6, 95.9]],
    }
    assert b._lv1_kernel(tune, "f32", 0) == "k_ic_apply_blk<float,0,0>"
    assert b._lv1_kernel(tune, "f32", 1) == "k_ic_apply<float,1,1>"
    assert b._lv1_kernel(tune, "f64", 0) == "k_ic_apply_stg<double,0,0>"
    assert b._lv1_kernel(tune, "f64", 1) == "k_ic_apply_blk<double,1,1>"  # b2: last candidate is blocked 256
    # no tuned level-1 shape (tuning off): the natural-order kernel
    assert b._lv1_kernel({}, "f32", 1) == "k_ic_apply<float,1,1>"
