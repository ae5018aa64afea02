"""Writes config4_digests.json: the SHA-256 digest (words, level, scale bits) of every
ciphertext of one encrypted training step at config 4's full size, computed by the oracle's
CPU evaluator (the restated reference Evaluator behind the HeOps methods). The GPU test
`tests/test_gpu_nn.py::test_config4_ct_for_ct` runs the same step from the same seeded keys,
ciphertexts and data on the device and compares every digest.

Config 4: n16_train (N = 2^16, 58 + 31 x 42-bit q, 4 x 58-bit p, dnum 8, scale 2^42),
Layout(2^15, 256, 64), 196 -> 64 -> 10 with Square, B = 64, inputs U[0, 1), weights and
biases U[-0.1, 0.1) (numpy default_rng(43)), keys from KeyGenerator seed 41 (8 generators),
client encryptions seeded 2, 3, ... (symmetric, as the other training tests), lr 0.05.

Run from the repository root: python tests/golden/make_config4_digests.py (about half an
hour on 8 cores; the keys take about 15 GB of host memory).
"""

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from conftest import load_package  # noqa: E402
from nn_backends import Client, OracleHeOps, ct_digest, deterministic_keys, step_values  # noqa: E402
from test_nn import encrypt_network, make_problem  # noqa: E402

import oracle as O  # noqa: E402

N16_TRAIN = dict(log_n=16, q_bits=[58] + [42] * 31, p_bits=[58] * 4, scale_bits=42, dnum=8)


def main():
    nn = load_package().nn
    ps = N16_TRAIN
    P = O.Params.from_bits(ps["log_n"], ps["q_bits"], ps["p_bits"], ps["scale_bits"], ps["dnum"])
    layout, dims = nn.Layout(P.n // 2, 256, 64), [196, 64, 10]
    t0 = time.time()
    kg, rk, gk = deterministic_keys(P, nn.mlp_rotation_steps(dims, layout), 41)
    print(f"keys: {len(gk)} Galois + relin, {time.time() - t0:.0f} s", flush=True)
    cpu = OracleHeOps(P, rk, gk)
    client = Client(P, kg)
    ws, bs, x, y = make_problem(nn, dims, layout, 43)
    top, delta = P.max_level, float(2.0 ** ps["scale_bits"])
    mlp, xc, yc = encrypt_network(nn, client, cpu.ev, cpu, layout, dims, ws, bs, x, y, top, delta, cpu._w)
    t0 = time.time()
    tr = nn.Trainer(cpu, layout, [nn.Sgd(0.05) for _ in dims[1:]])
    v = tr.train_batch(mlp, xc, yc)
    print(f"step: {time.time() - t0:.0f} s", flush=True)
    out = {
        "config": "n16_train, Layout(2^15, 256, 64), 196-64-10 Square, B 64, keys seed 41 (8 generators), "
                  "data default_rng(43), lr 0.05",
        "counter": cpu.counter(),
        "trace": [list(t) for t in tr.trace],
        "values": [[name, ct.level(), ct.scale(), ct_digest(ct.ct.data(), ct.level(), ct.scale())]
                   for name, ct in step_values(v, mlp)],
    }
    with open(os.path.join(HERE, "config4_digests.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"{len(out['values'])} digests written", flush=True)


if __name__ == "__main__":
    main()
