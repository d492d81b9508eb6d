"""Regenerates tests/golden/gen_index_sha256.json from the reference binary.

Runs the reference T-BLAEQ built from source by `make -C oracle ref` (oracle/_ref/T-BLAEQ) with
`--gen-index` for each case below and records the SHA-256 of every file it writes. The tests then
check that the B200 build's generator and serializer write the same bytes without needing the
reference at test time.

usage: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(REPO, "oracle", "_ref", "T-BLAEQ")

# (name, N, D, height, ratios, seed, sigma divisor, extra flags)
CASES = [
    ("small_cfg", 500000, 5, 4, "80,40,20", 20260330, 2.2, []),
    ("d3_tiny", 20000, 3, 4, "10,10,10", 7, 3.0, []),
    ("d8_mid", 200000, 8, 4, "100,50,20", 1, 3.0, []),
    ("d16_mid", 100000, 16, 4, "100,50,20", 2, 2.5, []),
    ("truncated", 3000, 2, 4, "10,20,30", 5, 3.0, []),
    ("int_h3", 5000, 4, 3, "7,9", 11, 1.5, ["--gen-int"]),
    ("uneven", 12345, 6, 4, "7,3,5", 99, 4.0, []),
    ("trunc_drop", 1000, 3, 5, "10,10,10,10", 3, 3.0, []),
]


def sha_dir(d):
    return {f: hashlib.sha256(open(os.path.join(d, f), "rb").read()).hexdigest() for f in sorted(os.listdir(d))}


def main():
    if not os.path.exists(REF_BIN):
        sys.exit(f"{REF_BIN} missing: run `make -C oracle ref` where the reference sources are mounted")
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, N, D, height, ratios, seed, sdiv, extra in CASES:
            d = os.path.join(tmp, name)
            cmd = [REF_BIN, "--gen-index", "-i", d, "--gen-N", str(N), "--gen-D", str(D), "--height", str(height),
                   "--ratios", ratios, "--gen-seed", str(seed), "--gen-sigma-divisor", str(sdiv)] + extra
            subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
            out[name] = {"params": {"N": N, "D": D, "height": height, "ratios": [int(r) for r in ratios.split(",")],
                                    "seed": seed, "sigma_divisor": sdiv, "is_int": "--gen-int" in extra},
                         "sha256": sha_dir(d)}
    with open(os.path.join(HERE, "gen_index_sha256.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", len(out), "cases")


if __name__ == "__main__":
    main()
