"""Generate tests/golden/peaks_golden.json.

The cases restate the peak finder's unit tests in the reference
(rust/src/peaks.rs:290-371): the same inputs, the same (n_peaks,
min_distance, use_max), and the outputs those tests assert.  Where a
reference test asserts only a property (chunked == single pass), the
expected output recorded here is the single-pass result, which that test
pins as the answer.

Run from the repository root:  python tests/golden/make_peaks_golden.py
"""

import json
import math
import os
import struct


def f32(x):
    return struct.unpack("f", struct.pack("f", x))[0]


def case(name, data, n_peaks, min_distance, use_max, idx, val, source):
    return {
        "name": name,
        "data": [f32(v) for v in data],
        "n_peaks": n_peaks,
        "min_distance": min_distance,
        "use_max": use_max,
        "expect_idx": idx,
        "expect_val": [f32(v) for v in val] if val is not None else None,
        "source": source,
    }


def main():
    cases = []
    # peaks.rs:290-298 single_peak
    cases.append(case("single_peak", [0.0, 1.0, 3.0, 1.0, 0.0], 32, 1, True, [2], [3.0],
                      "rust/src/peaks.rs:290-298"))
    # peaks.rs:300-307 single_minimum
    cases.append(case("single_minimum", [5.0, 3.0, 1.0, 3.0, 5.0], 32, 1, False, [2], [1.0],
                      "rust/src/peaks.rs:300-307"))
    # peaks.rs:309-321 distance_constraint
    cases.append(case("distance_constraint", [0.0, 5.0, 0.0, 4.0, 0.0, 0.0, 0.0, 0.0, 3.0, 0.0],
                      32, 4, True, [1, 8], [5.0, 3.0], "rust/src/peaks.rs:309-321"))
    # peaks.rs:323-335 respects_n_peaks_limit: data[i] = i/10 at i = 1, 11, ...,
    # 191; top 5 are 191, 181, 171, 161, 151 (values strictly decreasing).
    data = [0.0] * 200
    for i in range(1, 200, 10):
        data[i] = f32(i) / f32(10.0)
    top = [191, 181, 171, 161, 151]
    cases.append(case("respects_n_peaks_limit", data, 5, 1, True, top,
                      [f32(f32(i) / f32(10.0)) for i in top], "rust/src/peaks.rs:323-335"))
    # peaks.rs:337-355 chunked_matches_single_pass: sin(0.3 i), n_peaks 8,
    # min_distance 3, maxima.  The single-pass answer: every local maximum of
    # sin(0.3 i) on 0..99 (period ~20.94 samples) is ~1; the greedy keeps them
    # all (they are > 3 apart) up to 8, best first.
    data = [f32(math.sin(f32(i) * f32(0.3))) for i in range(100)]
    cases.append(case("chunked_matches_single_pass", data, 8, 3, True, None, None,
                      "rust/src/peaks.rs:337-355"))
    # peaks.rs:357-362 empty_data
    cases.append(case("empty_data", [], 32, 1, True, [], [], "rust/src/peaks.rs:357-362"))
    # peaks.rs:364-370 monotonic_no_peaks
    cases.append(case("monotonic_no_peaks", [float(i) for i in range(50)], 32, 1, True, [],
                      [], "rust/src/peaks.rs:364-370"))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "peaks_golden.json")
    with open(out, "w") as fh:
        json.dump({"generator": "tests/golden/make_peaks_golden.py", "cases": cases}, fh,
                  indent=1)
    print(f"wrote {out} ({len(cases)} cases)")


if __name__ == "__main__":
    main()
