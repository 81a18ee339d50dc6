"""Generates the known-answer vectors in tests/golden/kat.json.

The reference publishes no numeric fixtures, so these vectors are computed here by independent
pure-Python / numpy implementations of the published formulas the reference uses:
  * the PCG-style hash and unit float of src/importance_sampling/shared.wesl:266-284
    (Python integers modulo 2^32; f32(u) * 2^-32 via numpy float32);
  * IEEE binary16 packing (numpy float16, round to nearest even) and bfloat16 packing
    (round to nearest even on the f32 bit pattern) used by Material::new (src/lib.rs:96-182);
  * WGSL pack2x16snorm of the octahedral normal encoding (general.wesl:1293-1305).
Run: python tests/golden/make_golden.py
"""
import json
import os

import numpy as np

M32 = 0xFFFFFFFF


def rand_u32(s):
    state = (s * 747796405 + 2891336453) & M32
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M32
    return ((word >> 22) ^ word) & M32


def rand_f32(s):
    x = np.float32(np.float32(rand_u32(s)) * np.float32(2.0 ** -32))
    return float(x - np.floor(x))


def f16_bits(x):
    return int(np.array([x], dtype=np.float32).astype(np.float16).view(np.uint16)[0])


def bf16_bits(x):
    b = int(np.array([x], dtype=np.float32).view(np.uint32)[0])
    if (b & 0x7FFFFFFF) > 0x7F800000:
        return (b >> 16) | 0x40
    lsb = (b >> 16) & 1
    return ((b + 0x7FFF + lsb) >> 16) & 0xFFFF


def snorm16(v):
    c = min(1.0, max(-1.0, float(np.float32(v))))
    return int(np.floor(np.float32(0.5) + np.float32(32767.0) * np.float32(c))) & 0xFFFF


def octa(n):
    n = np.asarray(n, np.float32)
    s = max(float(np.abs(n).sum()), 0.01)
    v = n / np.float32(s)
    if v[1] >= 0:
        return snorm16(v[0]) | (snorm16(v[2]) << 16)
    xx = np.copysign(1.0 - abs(v[2]), v[0]) if v[0] < 0 else abs(1.0 - abs(v[2]))
    zz = np.copysign(1.0 - abs(v[0]), v[2]) if v[2] < 0 else abs(1.0 - abs(v[0]))
    return snorm16(xx) | (snorm16(zz) << 16)


def main():
    rng = np.random.default_rng(7)
    seeds = [0, 1, 2, 3, 12345, 0x7FFFFFFF, 0xFFFFFFFF] + [int(x) for x in rng.integers(0, 2 ** 32, 57, dtype=np.uint64)]
    floats = [0.0, -0.0, 1.0, -1.0, 0.5, 1.5, 2.4063, 2.4922, 1.00027531, 65504.0, 65520.0, 1e-8, 6.1e-5, 5.96e-8,
              3.0e-8, 100.0, 15.0, 0.3, 1.0 / 3.0, 1e30] + [float(x) for x in rng.normal(0, 10, 30)]
    normals = [[0, 1, 0], [0, -1, 0], [1, 0, 0], [-1, 0, 0], [0, 0, 1], [0, 0, -1]]
    normals += [list(map(float, v / np.linalg.norm(v))) for v in rng.normal(size=(30, 3))]
    out = {
        "rand_u32": [[s, rand_u32(s)] for s in seeds],
        "rand_f32": [[s, rand_f32(s)] for s in seeds],
        "f16": [[f, f16_bits(f)] for f in floats],
        "bf16": [[f, bf16_bits(f)] for f in floats],
        "octahedral": [[n, octa(n)] for n in normals],
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kat.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", path)


if __name__ == "__main__":
    main()
