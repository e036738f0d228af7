"""Extract the known-answer vectors of the reference's own unit tests for the
rasterizer path and write them, with their expected outputs, to
reference_known_answers.json.

Run from the repository root with the reference checkout at hand:
    python tests/golden/make_golden.py /path/to/RustScan
The expected outputs are computed by the rule each reference test asserts
(stable argsort by (key, index), inclusive scan, identity of degree-0 SH on
rgb_to_sh0 values, projection of (0,0,1) to the principal point). The JSON is
committed; tests read only the JSON.
"""
import json
import os
import re
import sys


def rust_arrays(text, fn_name):
    """Literal u32 arrays passed in the body of `fn fn_name`."""
    m = re.search(r"fn\s+" + re.escape(fn_name) + r"\s*\(\)\s*\{(.*?)\n\}", text, re.S)
    if not m:
        raise SystemExit(f"test {fn_name} not found")
    body = m.group(1)
    return [[int(x) for x in arr.split(",") if x.strip()] for arr in re.findall(r"&\[([0-9,\s]*)\]", body)], body


def _concat_text(body):
    """The text of the first concat!(...) of string literals in a test body."""
    m = re.search(r"concat!\((.*?)\n\s*\)", body, re.S)
    parts = re.findall(r'"((?:[^"\\]|\\.)*)"', m.group(1))
    return "".join(p.encode().decode("unicode_escape") for p in parts)


def scene_file_cases(ref):
    """Files the reference's scene reader is tested on (RustGS/src/io/scene_io/tests.rs),
    with the values those tests assert after loading."""
    src = open(os.path.join(ref, "RustGS/src/io/scene_io/tests.rs")).read()

    def body(name):
        m = re.search(r"fn\s+" + name + r"\s*\(\)\s*\{(.*?)\n\}", src, re.S)
        if not m:
            raise SystemExit(f"test {name} not found")
        return m.group(1)

    cases = []
    b = body("test_load_external_raw_logit_opacity")
    cases.append({"test": "test_load_external_raw_logit_opacity", "ascii": _concat_text(b),
                  "expected": {"opacity_logit": [float(re.search(r"opacity_logit\(0\) - ([0-9.]+)", b).group(1))]}})
    b = body("test_load_external_channel_major_sh_coeffs")
    sh = [float(x) for x in re.search(r"sh_coeffs,\s*&\[([^\]]*)\]", b).group(1).split(",")]
    cases.append({"test": "test_load_external_channel_major_sh_coeffs", "ascii": _concat_text(b),
                  "expected": {"sh_degree": int(re.search(r"sh_degree, (\d+)", b).group(1)), "sh_coeffs": sh}})
    b = body("test_load_binary_brush_export_ply")
    header = _concat_text(b)
    head = re.search(r"let mut row = vec!\[(.*?)\];", b, re.S).group(1)
    consts = {"-std::f32::consts::LN_10": -2.302585092994046}
    row = []
    for tok in [t.strip() for t in head.split(",") if t.strip()]:
        row.append(consts[tok] if tok in consts else float(tok.replace("f32", "")))
    lo, hi = (int(x) for x in re.search(r"row\.extend\(\((\d+)\.\.=(\d+)\)", b).groups())
    row += [float(v) for v in range(lo, hi + 1)]
    # The test's expectation: DC, then per coefficient the three channels of
    # the channel-major f_rest block (coeff k: k+1, k+16, k+31).
    exp_sh = [0.1, 0.2, 0.3]
    for k in range(15):
        exp_sh += [float(k + 1), float(k + 16), float(k + 31)]
    cases.append({"test": "test_load_binary_brush_export_ply", "binary_header": header, "row_f32": row,
                  "expected": {"sh_degree": int(re.search(r"sh_degree, (\d+)", b).group(1)),
                               "position": [1.0, 2.0, 3.0], "opacity_logit": [2.0], "sh_coeffs": exp_sh}})
    return cases


def main(ref):
    gp = os.path.join(ref, "RustGS/src/training/gpu_primitives")
    sort_src = open(os.path.join(gp, "radix_sort/tests.rs")).read()
    scan_src = open(os.path.join(gp, "prefix_sum/tests.rs")).read()
    out = {"source": "RustGS/src/training/gpu_primitives/{radix_sort,prefix_sum}/tests.rs, RustGS/src/sh/tests.rs, "
                     "RustGS/src/core/camera_tests.rs, RustGS/src/training/backward/rasterize_bwd/tests.rs, "
                     "RustGS/src/io/scene_io/tests.rs"}
    argsort = []
    for name in ["test_radix_sort_empty", "test_radix_sort_single", "test_radix_sort_small",
                 "test_radix_sort_power_of_two"]:
        arrs, _ = rust_arrays(sort_src, name)
        keys = arrs[0]
        argsort.append({"test": name, "keys": keys,
                        "expected": sorted(range(len(keys)), key=lambda i: (keys[i], i))})
    # test_radix_sort_large: (0..513).map(|index| ((index * 37) % 101))
    _, body = rust_arrays(sort_src, "test_radix_sort_large")
    mm = re.search(r"\(0\.\.(\d+)\)\.map\(\|index\| \(\(index \* (\d+)\) % (\d+)\)", body)
    n, mul, mod = (int(g) for g in mm.groups())
    keys = [(i * mul) % mod for i in range(n)]
    argsort.append({"test": "test_radix_sort_large", "keys": keys,
                    "expected": sorted(range(n), key=lambda i: (keys[i], i))})
    out["argsort"] = argsort
    arrs, _ = rust_arrays(sort_src, "test_radix_sort_by_key_small")
    k, v = arrs
    order = sorted(range(len(k)), key=lambda i: (k[i], i))
    out["sort_by_key"] = [{"test": "test_radix_sort_by_key_small", "keys": k, "values": v,
                           "expected_keys": [k[i] for i in order], "expected_values": [v[i] for i in order]}]
    scans = []
    for name in ["test_prefix_sum_empty", "test_prefix_sum_single", "test_prefix_sum_power_of_two",
                 "test_prefix_sum_non_power_of_two"]:
        arrs, _ = rust_arrays(scan_src, name)
        x = arrs[0]
        acc, exp = 0, []
        for a in x:
            acc += a
            exp.append(acc)
        scans.append({"test": name, "input": x, "expected": exp})
    out["prefix_sum"] = scans
    sh_src = open(os.path.join(ref, "RustGS/src/sh/tests.rs")).read()
    rgb = [float(x) for x in re.search(r"let rgb = \[([^\]]*)\]", sh_src).group(1).split(",")]
    out["sh_degree0_identity"] = {"rgb": rgb, "viewdir": [0.0, 0.0, 1.0]}
    cam_src = open(os.path.join(ref, "RustGS/src/core/camera_tests.rs")).read()
    f, w, h = re.search(r"Intrinsics::from_focal\(([0-9.]+), (\d+), (\d+)\)", cam_src).groups()
    out["camera_project"] = {"focal": float(f), "width": int(w), "height": int(h), "point": [0.0, 0.0, 1.0],
                             "expected_pixel": [int(w) / 2, int(h) / 2], "tolerance": 1.0}
    # backward/rasterize_bwd/tests.rs:6-54: a single projected splat in one 16x16 tile.
    bwd_src = open(os.path.join(ref, "RustGS/src/training/backward/rasterize_bwd/tests.rs")).read()
    vals = re.search(r"vec!\[([0-9.,\sf32]*)\]", bwd_src).group(1).replace("f32", "")
    out["single_splat_backward"] = {"projected": [float(x) for x in vals.split(",") if x.strip()],
                                    "image": [16, 16], "upstream": "ones"}
    out["scene_files"] = scene_file_cases(ref)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_known_answers.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the RustScan checkout>")
    main(sys.argv[1])
