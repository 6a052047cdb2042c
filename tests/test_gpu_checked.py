"""The checked build (libumapcu_checked.so, the same sources compiled with
UMAPCU_CHECKED): on the device every CSR offset, other endpoint, injected
negative and schedule record is bounds-checked before use; a bad one is
skipped -- the access is never made -- and the call returns UMAPCU_BAD_ARG.
The malformed inputs go only to the checked library, through the one entry
point whose CSR lives in caller memory (umapcu_optimise_csr_noalloc), in a
child process that loads the checked library in place of the plain one
(needs a B200). The whole GPU suite also passes against the checked library
(UMAPCU_LIB=.../libumapcu_checked.so)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "manifolds-rs_b200", "umapcu", "libumapcu_checked.so")

_CHILD = r"""
import ctypes as C, json, sys
import numpy as np
import torch
sys.path[:0] = [ROOT, ROOT + "/manifolds-rs_b200"]
import umapcu
import umapdata.synth as S
assert "checked" in umapcu.version(), umapcu.version()
X, _ = S.isotropic_mixture(2500, 20, 6, seed=3)
idx, dist = umapcu.knn_exact(X, 15)
g = umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), 40)
adj = umapcu.coo_to_adjacency_list(g)
init = umapcu.random_layout(2500, 2, 9)
p = umapcu.UmapOptimParams(n_epochs=40)
want = init.copy()
umapcu.optimise_embedding_adam_gpu(want, adj, p, seed=5)
st = umapcu.UmapGpuState(init, adj, p, None, 5)
csr = st.csr()
st.close()
period = csr["eps"][csr["edge_idx"]].astype(np.float32)
n, ne = 2500, int(period.size)
fn = umapcu.lib().umapcu_optimise_csr_noalloc
fn.restype = C.c_int
fn.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
               C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]
cp = p._c()
dev = torch.device("cuda")
d_per = torch.from_numpy(period).to(dev)
def call(offsets, other):
    d_y = torch.from_numpy(init.copy()).to(dev)
    d_off = torch.from_numpy(offsets.view(np.int32)).to(dev)
    d_oth = torch.from_numpy(other.view(np.int32)).to(dev)
    torch.cuda.synchronize()
    rc = fn(d_y.data_ptr(), n, 2, d_off.data_ptr(), d_oth.data_ptr(), d_per.data_ptr(), ne, C.byref(cp), 5, 0, None)
    torch.cuda.synchronize()
    return rc, d_y.cpu().numpy()
out = {}
rc, y = call(csr["offsets"], csr["other"])
out["valid"] = [rc, bool(np.array_equal(y, want))]
bad = csr["other"].copy(); bad[[7, 1000, ne - 1]] = n + 7
out["other_out_of_range"] = call(csr["offsets"], bad)[0]
off = csr["offsets"].copy(); off[n] = ne + 64
out["offset_past_entries"] = call(off, csr["other"])[0]
off = csr["offsets"].copy(); off[100], off[101] = off[101], off[100] + 1
out["offsets_out_of_order"] = call(off, csr["other"])[0]
rc, y = call(csr["offsets"], csr["other"])
out["valid_after"] = [rc, bool(np.array_equal(y, want))]
print(json.dumps(out))
"""


def test_checked_build_refuses_malformed_csr():
    assert os.path.exists(CHECKED), "checked library not built"
    env = dict(os.environ, UMAPCU_LIB=CHECKED)
    r = subprocess.run([sys.executable, "-c", _CHILD.replace("ROOT", repr(ROOT))], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    OK, BAD_ARG = 0, 7
    assert out["valid"] == [OK, True] and out["valid_after"] == [OK, True], out
    for k in ("other_out_of_range", "offset_past_entries", "offsets_out_of_order"):
        assert out[k] == BAD_ARG, (k, out)
