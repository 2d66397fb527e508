"""The oracle as a self-contained CPU solve (no GPU): it builds its own mesh
and seeded initial state with the host mesh builder compiled into
``liboracle.so``, maps no other library, and its zone-parallel loops give
the same bits on any number of host threads."""
import os
import subprocess
import sys

import numpy as np

import cubesphere_b200 as cs
from oracle import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_standalone_oracle_builds_the_library_mesh_and_state():
    pr = cs.preset("shell16")
    o = Oracle(params=cs.make_params(**pr["params"]))
    o.init_problem(cs.make_init(**pr["init"]))
    s = cs.Solve(**pr["params"])
    s.mesh_build(device=False)
    st = s.init_problem_host(**pr["init"])
    for f in range(len(cs.GEOM_FIELDS)):
        assert np.array_equal(o.geometry(f), s.geometry(f)), cs.GEOM_FIELDS[f]
    m, stn = o.mask_stencil()
    assert np.array_equal(m, s.mask()) and np.array_equal(stn, s.stencil())
    got = o.get_state()
    for k in st:
        assert np.array_equal(got[k], st[k]), k
    o.close()
    s.close()


_CHILD = r"""
import hashlib, sys
sys.path.insert(0, {root!r})
import cubesphere_b200 as cs
from oracle import Oracle
pr = cs.preset("shell16")
o = Oracle(params=cs.make_params(**pr["params"]))
o.init_problem(cs.make_init(**pr["init"]))
dt = o.evaluate_timestep(1e30)
dt = o.step(dt)
h = hashlib.sha256()
st = o.get_state()
for k in ("U", "ent", "bxf", "byf", "bzf"):
    h.update(st[k].tobytes())
h.update(repr(dt).encode())
maps = open("/proc/self/maps").read()
print(h.hexdigest(), "libcubesphere_b200" in maps, "liboracle" in maps)
"""


def _child(threads: int) -> list:
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([sys.executable, "-c", _CHILD.format(root=ROOT)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout.split()


def test_zone_parallel_oracle_is_thread_count_independent_and_self_contained():
    """One IMEX-RK2 step of shell16 on 1 and on 4 host threads: the same
    state and time step bit for bit; the process never maps the CUDA
    library (the CPU reference arm of the bench runs this way)."""
    one, four = _child(1), _child(4)
    assert one[0] == four[0]
    assert one[1] == "False" and four[1] == "False"
    assert one[2] == "True"
