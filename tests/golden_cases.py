"""Loader for the golden fixtures recorded from the compiled reference."""
import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def system(name):
    from hfps import workloads
    spec = dict(index()[name]["spec"])
    cfg = spec.pop("config")
    if "n" in spec:
        spec["n"] = tuple(spec["n"])
    return workloads.make(cfg, **spec)


def policy(name):
    import ref_oracle
    return ref_oracle.MgPolicy(**index()[name]["policy"])


def arrays(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def probe(sys_):
    from hfps import workloads
    return np.ascontiguousarray(workloads.normals(99, sys_.cells).reshape(sys_.rhs.shape))


def digest(s):
    h = hashlib.sha256()
    for a in (s.diagonal, s.face_x, s.face_y, s.face_z, s.rhs, *s.faces):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    if s.active is not None:
        h.update(np.ascontiguousarray(s.active, dtype=np.uint8).tobytes())
    return h.hexdigest()
