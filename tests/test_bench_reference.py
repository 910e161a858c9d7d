"""The CPU arm of bench.py: same inputs and config as the GPU arm, without the product.

The oracle library carries its own build of the seeded workload generator, so the CPU
baseline makes the long pair without loading librfd.so; these checks need no GPU.
"""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_generator_equals_librfd_generator(built):
    import oracle
    for cfg, n in ((0, None), (2, 5), (4, 2)):
        a = oracle.gen_config(cfg, npairs=n) if n else oracle.gen_config(cfg)
        b = built.gen_config(cfg, npairs=n) if n else built.gen_config(cfg)
        for (p1, q1), (p2, q2) in zip(a, b):
            assert np.array_equal(p1, p2) and np.array_equal(q1, q2)
    p, q = oracle.gen_config_pair(2, 11)
    p2, q2 = built.gen_config(2, npairs=12)[11]
    assert np.array_equal(p, p2) and np.array_equal(q, q2)


def test_reference_arm_loads_only_the_oracle(built):
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', "
            "'--warmup', '0', '--points', '600', '--cpu-sample', '300']\n"
            "import bench; bench.main()\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('LIBS', 'librfd' in maps, 'liboracle' in maps)\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=300, check=True).stdout.splitlines()
    line = json.loads(out[0])
    assert out[-1] == "LIBS False True"
    assert line["impl"] == "reference" and line["unit"] == "solves/s"
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.config_dict(600, 600, 600, 3, 1)
    assert line["e2e"]["h2d_bytes_per_step"] == 0
