"""Write tests/golden/kats.json: the known answers and tolerances that the
reference's own checks hold for this path, with the file:line of each.

Run from the repository root as `python tests/golden/make_kats.py [REFERENCE]`,
where REFERENCE is the reference project's root (or set RADIX_REFERENCE).
When it is given and present, every cited line is read and checked to contain
the quoted text, so the fixture cannot drift from its source.
"""
import json
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RADIX_REFERENCE", "")
HERE = os.path.dirname(os.path.abspath(__file__))

KATS = {
    "sort_keys_monotonic": {
        "source": "scripts/check-core.ts:1194-1208",
        "quote": [[1195, "const distances = [0, 1e-12, 1e-6, 0.001, 0.5, 1, 1.0001, 2, 100, 1e6, 1e12, 3e38];"],
                  [1203, "[Infinity, NaN, -Infinity].some((d) => SortKeys.compute(d, bits) !== SortKeys.invalid(bits))"],
                  [1207, "return SortKeys.compute(1, 32) !== (0xffffffff ^ 0x3f800000) >>> 0"]],
        "distances": [0, 1e-12, 1e-6, 0.001, 0.5, 1, 1.0001, 2, 100, 1e6, 1e12, 3e38],
        "non_finite": ["inf", "nan", "-inf"],
        "key_of_1_at_32": 0xFFFFFFFF ^ 0x3F800000,
    },
    "sort_stability": {
        "source": "scripts/check-core.ts:1210-1229",
        "quote": [[1211, "const count = 20000;"],
                  [1212, "(i % 97 === 0 ? Infinity : Math.round(random() * 1000) / 10)"]],
        "count": 20000, "infinite_every": 97, "step": 0.1, "max": 100.0,
    },
    "sh_band1": {
        "source": "scripts/check-core.ts:1666-1676",
        "quote": [[1668, "c[0] = 1;"], [1669, "c[4] = 2;"], [1670, "c[8] = 3;"], [1674, "const k = 0.4886025;"]],
        "coeff_index_value": [[0, 1.0], [4, 2.0], [8, 3.0]],
        "k": 0.4886025,
        "expect": [["y", 0, -1.0], ["z", 1, 2.0], ["x", 2, -3.0]],
        "tolerance": 1e-9,
    },
    "sh_legendre": {
        "source": "scripts/check-core.ts:1704-1722",
        "quote": [[1707, "for (let n = 0; n < 200; n += 1) {"], [1721, "return worst < 2e-6 ?"]],
        "directions": 200, "tolerance": 2e-6,
    },
    "ext_budgets": {
        "source": "scripts/check-core.ts:341-400",
        "quote": [[355, "if (Math.abs(out.opacity - s.opacity) > 1 / 256 + 1e-12) {"],
                  [364, "> maxAbs / 255 + 1e-9) {"],
                  [375, "degrees(rotation) <= 0.45"],
                  [391, "return degrees(worst) <= 0.03"]],
        "opacity": 1.0 / 256, "rgb_of_max": 1.0 / 255, "rotation_degrees": 0.45, "small_turn_degrees": 0.03,
    },
    "identity_quat": {
        "source": "scripts/check-core.ts:394-400",
        "quote": [[399, "out.x === 0 && out.y === 0 && out.z === 0 && out.w === 1"]],
    },
    "sort_grid": {
        "source": "test/gpu/renderTests.ts:31-57",
        "quote": [[35, "for (const count of [0, 1, 4095, 4096, 4097, 70000]) {"]],
        "counts": [0, 1, 4095, 4096, 4097, 70000], "bits": [16, 24, 32],
    },
    "compact_then_sort": {
        "source": "test/gpu/renderTests.ts:59-90",
        "quote": [[62, "const count = 20000;"], [63, "(random() < 0.3 ? SortKeys.invalid(bits)"]],
        "count": 20000, "invalid_fraction": 0.3,
    },
    "ewa_bound": {
        "source": "test/gpu/renderTests.ts:242-277",
        "quote": [[272, "Math.abs(bound.scales[0] / major - 1) > 0.01 || Math.abs(bound.scales[1] / minor - 1) > 0.02"]],
        "splats": 200, "blur_amount": 0, "major_tolerance": 0.01, "minor_tolerance": 0.02,
        "camera": {"fov": 60, "near": 0.1, "far": 100, "width": 128, "height": 64, "position": [-0.03, 0, 0]},
    },
    "culling": {
        "source": "test/gpu/renderTests.ts:302-321",
        "quote": [[303, "const cases = [splat([0, 0, -3], 0.1), splat([0, 0, 3], 0.1), splat([40, 0, -3], 0.1), splat([0, 0, -3], 0.1, [1, 1, 1], 0.001)];"],
                  [309, "if (culled.join() !== \"false,true,true,true\") {"],
                  [313, "const expected = cullKeys ? \"false,true,true,true\" : \"false,false,false,true\";"]],
        "centers": [[0, 0, -3], [0, 0, 3], [40, 0, -3], [0, 0, -3]], "scale": 0.1, "opacities": [1, 1, 1, 0.001],
        "culled": [False, True, True, True],
        "invalid_cull_keys": [False, True, True, True], "invalid_no_cull_keys": [False, False, False, True],
    },
    "key_tolerance_fp32_distance": {
        "source": "test/gpu/renderTests.ts:323-339",
        "quote": [[332, "if (Math.abs(keys[i] - expected) > (bits === 32 ? 4 : 1)) {"]],
        "tolerance": {"16": 1, "24": 1, "32": 4},
    },
    "sort_guard": {
        "source": "test/gpu/renderTests.ts:341-367",
        "quote": [[344, "const splats = [splat([0, 0, -4], 0.05, [1, 1, 1], 1), splat([5.5, 0, -4], 0.05, [1, 1, 1], 1), splat([20, 0, -4], 0.05, [1, 1, 1], 1), splat([0, 0, 4], 0.05, [1, 1, 1], 1)];"],
                  [361, "return guarded.join() === \"true,true,false,false\""]],
        "centers": [[0, 0, -4], [5.5, 0, -4], [20, 0, -4], [0, 0, 4]], "scale": 0.05, "guard": 0.5,
        "valid_guard0": [True, True, True, True], "valid_guard": [True, True, False, False],
        "camera": {"fov": 60, "near": 0.1, "far": 100, "width": 128, "height": 64, "position": [0, 0, 0]},
    },
    "codecs_depth_angle": {
        "source": "test/gpu/splatTests.ts:589-612",
        "quote": [[601, "if (!(Math.abs(back / expected - 1) <= 2 ** -16 * 1.01)) {"],
                  [605, "(Math.PI / 8192) * 1.01"]],
        "depth_rel": 2.0 ** -16, "angle": 3.141592653589793 / 8192,
    },
    "sort_key_alignment": {
        "source": "src/core/layout.ts:26-29,70-72",
        "quote": [[26, "static readonly WIDTH = 1024;"], [27, "static readonly MAX_PACKING = 4;"]],
        "row_elements": 4096,
    },
}


def verify():
    bad = []
    for name, k in KATS.items():
        path = os.path.join(REF, k["source"].split(":")[0])
        with open(path) as f:
            lines = f.read().split("\n")
        for line, text in k["quote"]:
            if text not in lines[line - 1]:
                bad.append(f"{name}: {k['source']} line {line} lacks {text!r}")
    return bad


if __name__ == "__main__":
    if os.path.isdir(REF):
        problems = verify()
        if problems:
            print("\n".join(problems))
            sys.exit(1)
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(KATS, f, indent=1)
    print("wrote kats.json")
