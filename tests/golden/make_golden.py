"""Regenerates tests/golden/reference_pins.json from the reference's own CPU
code, built from its sources by oracle/build_ref.sh into oracle/_ref/:

  * ref_ranlux: the reference host RANLUX (random/random.cpp,
    PRNG::initialize_CPU + produce_CPU) -- the stream the reference assigns
    to generator instance 0, for several RANDSERIES and luxury levels;
  * ref_cpurun: the reference sequential heatbath (SU(N)/suncpp) in its
    deterministic INTS=2 mode -- plaquettes of the closed-form start and
    after each sweep.

Usage: python tests/golden/make_golden.py   (needs oracle/_ref built)
"""
import json
import os
import struct
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")


def f32_bits(x):
    return struct.unpack("<I", struct.pack("<f", x))[0]


def ranlux_stream(series, lux, n):
    out = subprocess.check_output([os.path.join(REF, "ref_ranlux"), str(series), str(lux), str(n)]).decode().split()
    jseed = int(out[1])
    vals = [f32_bits(float.fromhex(x)) for x in out[4:]]
    return jseed, vals


def gid_plaquettes(group, dims, beta, sweeps):
    args = [os.path.join(REF, "ref_cpurun"), "plaq", str(group)] + [str(d) for d in dims] + \
        [repr(beta), "2", "54", str(sweeps)]
    rows = []
    for line in subprocess.check_output(args).decode().split("\n"):
        if line.strip():
            s, sp, tp, tot = line.split()
            rows.append([int(s), float(sp), float(tp), float(tot)])
    return rows


def main():
    pins = {"ranlux": [], "gid": []}
    for series, lux in [(54, 3), (1, 3), (12345, 4), (54, 2), (777, 0), (2024, 1)]:
        jseed, vals = ranlux_stream(series, lux, 1000)
        pins["ranlux"].append({"randseries": series, "luxury": lux, "jseed": jseed, "bits": vals})
    for group, dims, beta in [(3, (4, 4, 4, 4), 6.0), (2, (4, 4, 4, 4), 2.3), (3, (4, 6, 4, 2), 5.7),
                              (2, (6, 4, 2, 4), 2.3)]:
        pins["gid"].append({"group": group, "dims": list(dims), "beta": beta,
                            "rows": gid_plaquettes(group, dims, beta, 3)})
    with open(os.path.join(HERE, "reference_pins.json"), "w") as f:
        json.dump(pins, f, indent=0)


if __name__ == "__main__":
    main()
