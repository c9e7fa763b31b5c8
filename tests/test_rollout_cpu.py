"""Host side of the uneven-size rollout: the ctypes mirrors against the C
header, the tiler, the workload generator, the environment generator and the
entry point's argument validation (no GPU needed)."""

import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from pymdp_b200 import _lib


def _c_layout(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stddef.h>
#include <stdio.h>
#include "pymdp_b200.h"
#define F(T, m) printf(#T "." #m " %zu\\n", offsetof(T, m));
int main(void) {
  printf("b2_ro_agent %zu\\n", sizeof(b2_ro_agent));
  printf("b2_ro_tile %zu\\n", sizeof(b2_ro_tile));
  printf("b2_ro_buffers %zu\\n", sizeof(b2_ro_buffers));
  printf("b2_ro_config %zu\\n", sizeof(b2_ro_config));
  F(b2_ro_agent, S) F(b2_ro_agent, obs_mask) F(b2_ro_agent, ustride_r) F(b2_ro_agent, O) F(b2_ro_agent, dep) F(b2_ro_agent, dstride) F(b2_ro_agent, A_off) F(b2_ro_agent, C_off)
  F(b2_ro_agent, B_off) F(b2_ro_agent, D_off) F(b2_ro_agent, G_off) F(b2_ro_agent, gamma)
  F(b2_ro_buffers, Aprime_count) F(b2_ro_buffers, qs64) F(b2_ro_buffers, rec_G) F(b2_ro_buffers, sync_count)
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return dict((k, int(v)) for k, v in (line.split() for line in out.strip().splitlines()))


def test_ctypes_structs_match_header(tmp_path):
    c = _c_layout(tmp_path)
    assert c["b2_ro_agent"] == ctypes.sizeof(_lib.RoAgent)
    assert c["b2_ro_tile"] == ctypes.sizeof(_lib.RoTile)
    assert c["b2_ro_buffers"] == ctypes.sizeof(_lib.RoBuffers)
    assert c["b2_ro_config"] == ctypes.sizeof(_lib.RoConfig)
    for key, off in c.items():
        if "." in key:
            st, field = key.split(".")
            cls = {"b2_ro_agent": _lib.RoAgent, "b2_ro_buffers": _lib.RoBuffers}[st]
            assert getattr(cls, field).offset == off, key


def test_splitmix64_published_vector():
    from oracle.rollout import sm64, u01
    assert sm64(0) == 0xE220A8397B1DCDAF  # first output of SplitMix64 seeded with 0
    u = [float(u01(7, a, t, s)) for a in range(3) for t in range(3) for s in (0, 64, 128)]
    assert all(0.0 <= x < 1.0 for x in u) and len(set(u)) == len(u)


def test_categorical32_inverse_cdf():
    from oracle.rollout import categorical32
    p = np.array([0.0, 0.25, 0.0, 0.75], np.float32)
    assert categorical32(p, 0.0) == 1
    assert categorical32(p, 0.2499) == 1
    assert categorical32(p, 0.25) == 3
    assert categorical32(p, 0.9999999) == 3


def test_generator_respects_caps():
    from pymdp_b200.rollout import make_uneven_agents
    specs = make_uneven_agents(200, seed=3)
    for sp in specs:
        assert 1 <= len(sp.S) <= 4 and 1 <= len(sp.O) <= 6
        assert all(2 <= s <= 64 for s in sp.S) and all(2 <= o <= 32 for o in sp.O)
        assert all(1 <= u <= min(4, s) for u, s in zip(sp.U, sp.S))
        assert all(int(a[0].size) <= 4096 for a in sp.A)
        assert sp.num_policies <= 256 and 1 <= sp.policy_len <= 4
        for a in sp.A:
            np.testing.assert_allclose(a.sum(0), 1.0, rtol=1e-5)
        for b in sp.B:
            np.testing.assert_allclose(b.sum(0), 1.0, rtol=1e-5)


@pytest.mark.parametrize("cols", [1, 7, 16, 64])
def test_tiles_cover_every_policy_once(cols):
    from pymdp_b200.rollout import make_tiles, make_uneven_agents, tile_cost
    specs = make_uneven_agents(60, seed=4)
    tiles = make_tiles(specs, cols)
    cover = [np.zeros(sp.num_reduced_policies, np.int64) for sp in specs]
    for a, lo, hi, _ in tiles:
        assert 0 <= lo < hi <= specs[a].num_reduced_policies
        assert hi - lo <= cols and (hi - lo + 7) // 8 * 8 * sum(specs[a].S) <= _lib.RO_TAB_FLOATS
        cover[a][lo:hi] += 1
    assert all((c == 1).all() for c in cover)
    costs = [tile_cost(specs[a], lo, hi) for a, lo, hi, _ in tiles]
    assert costs == sorted(costs, reverse=True)


def _host_rollout(n=4):
    """Descriptors and fake (never dereferenced) buffer addresses."""
    from pymdp_b200.rollout import _descriptor, make_tiles, make_uneven_agents
    specs = make_uneven_agents(n, seed=5)
    descs = (_lib.RoAgent * n)()
    nA = nB = nC = nD = nll = nqs = nG = 0
    for i, sp in enumerate(specs):
        offs = {"A": [], "B": [], "C": []}
        for a in sp.A:
            offs["A"].append(nA)
            nA += (a.shape[0] + 1) * int(a[0].size)
            offs["C"].append(nC)
            nC += a.shape[0]
        for b in sp.B:
            offs["B"].append(nB)
            nB += b.size
        offs.update(D=nD, ll=nll, qs=nqs, G=nG)
        nD += sum(sp.S)
        nll += sum(int(a[0].size) for a in sp.A)
        nqs += sum(sp.S)
        nG += sp.num_policies
        descs[i] = _descriptor(sp, offs)
    tiles_np = np.ascontiguousarray(make_tiles(specs, 32))
    tiles = (_lib.RoTile * len(tiles_np))()
    ctypes.memmove(tiles, tiles_np.ctypes.data, tiles_np.nbytes)
    fake = 0x1000
    b = _lib.RoBuffers(fake, fake, fake, 0, nA, fake, nB, fake, nC, fake, nD, fake, nll, fake, fake, nqs, fake, nG,
                       fake, fake, 0, 0, 0, 0, 0, fake, 64)
    return descs, tiles, len(tiles_np), b


def _call(descs, tiles, n_tiles, b, steps=8, cfg=(256, 64, 32, 0)):
    lib = _lib.load()
    rc = lib.b2_rollout(None, ctypes.addressof(descs), len(descs), ctypes.addressof(tiles), n_tiles,
                        ctypes.byref(b), steps, 1, 16, 3, ctypes.byref(_lib.RoConfig(*cfg)))
    return rc, lib.b2_last_error().decode()


def test_rollout_validation_rejects_bad_input():
    descs, tiles, nt, b = _host_rollout()
    # a consistent input gets past validation (and fails only for want of a GPU)
    rc, msg = _call(descs, tiles, nt, b)
    assert rc in (_lib.B2_ERR_CUDA, _lib.B2_ERR_NO_DEVICE), msg
    rc, msg = _call(descs, tiles, nt, b, cfg=(192, 64, 32, 0))
    assert rc == _lib.B2_ERR_UNSUPPORTED and "threads" in msg
    rc, msg = _call(descs, tiles, nt, b, steps=40)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and "sync" in msg
    rc, msg = _call(descs, tiles, nt - 1, b)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and "cover" in msg
    d0 = descs[0]
    saved = d0.K[0]
    d0.K[0] = saved + 1
    rc, msg = _call(descs, tiles, nt, b)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and "K_m" in msg
    d0.K[0] = saved
    saved = d0.G_off
    d0.G_off = b.G_count
    rc, msg = _call(descs, tiles, nt, b)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and "G_off" in msg
    d0.G_off = saved
    tiles[0].p_hi = tiles[0].p_lo
    rc, msg = _call(descs, tiles, nt, b)
    assert rc == _lib.B2_ERR_INVALID_ARGUMENT and "tile" in msg


def test_reduced_policy_space():
    """Unobserved factors are dropped from the evaluated policy set; the map
    from a full policy to its reduced index keeps the observed actions."""
    from oracle.efe import construct_policies
    from pymdp_b200.rollout import AgentSpec, _descriptor
    rng = np.random.default_rng(0)
    S, U, T = [3, 4, 2], [2, 3, 2], 2
    A = [rng.dirichlet(np.ones(5), size=(3, 2)).transpose(2, 0, 1)]  # modality on factors 0 and 2
    B = [rng.dirichlet(np.ones(s), size=(s, u)).transpose(2, 0, 1) for s, u in zip(S, U)]
    sp = AgentSpec(A, B, [np.zeros(5)], [np.ones(s) / s for s in S], [[0, 2]], T)
    assert sp.observed == [0, 2] and sp.num_reduced_policies == 4 ** T and sp.num_policies == 12 ** T
    g = _descriptor(sp, {"A": [0], "C": [0], "B": [0, 0, 0], "D": 0, "ll": 0, "qs": 0, "G": 0})
    assert (g.obs_mask, g.n_multi_r, g.P_r, g.w0_r, list(g.ustride_r)[:3]) == (0b101, 4, 16, 4, [2, 0, 1])
    pol = construct_policies(S, U, T)
    red = construct_policies([S[0], S[2]], [U[0], U[2]], T)
    index = {tuple(r.reshape(-1)): i for i, r in enumerate(red)}
    for p, row in enumerate(pol):
        pr, W = 0, g.w0
        for t in range(T):
            mt = (p // W) % g.n_multi
            mr = sum(((mt // g.ustride[f]) % g.U[f]) * g.ustride_r[f] for f in range(3))
            pr = pr * g.n_multi_r + mr
            W //= g.n_multi
        assert pr == index[tuple(row[:, [0, 2]].reshape(-1))]
