"""Multicomponent species solves (vidyut.multicompsolves,
Source/Evolve.cpp:458-573; chunk checks Source/Vidyut.cpp:146-186).

Ions, then neutrals, are solved in chunks of comp_ion_chunks /
comp_neutral_chunks consecutive species, each chunk as one multigrid solve
(implicit_solve_scalar with numspec > 1, Source/ScalarSolve.cpp:540-875)
whose stopping test takes the max-norm over the chunk and whose bottom
BiCGStab sums its inner products over the chunk; background species of the
neutral range take part and are then reset to the step's starting value
before their own reactions.

CPU: the chunk arithmetic against a restatement of the reference's loops,
the Robin rule, and the oracle's joint solve against per-species solves
(the same solution to solver tolerance) and its multicomponent step against
the plain step.  GPU: the library's joint solve (one thread-block cluster
per chunk for the bottom solve) and its multicomponent steps against the
oracle, including background reactions with two correctors.
"""
import numpy as np
import pytest

import vidyut_b200 as vb
from oracle.oracle import Oracle
from vidyut_b200 import workloads as W
from vidyut_b200.compare import field_error

TIGHT = dict(linsolve_reltol=1e-13, linsolve_abstol=0.0)


def rel(a, b):
    return field_error(b, a)[1]


def ref_chunks(first, num, chunk):
    """The reference's chunk loops (Source/Evolve.cpp:462-495)."""
    out = []
    comp = first
    while comp <= first + num - chunk:
        out.append((comp, chunk))
        comp += chunk
    if comp != first + num:
        out.append((comp, first + num - comp))
    return out


@pytest.mark.parametrize("num,chunk", [(5, 5), (5, 2), (5, 3), (5, 1), (2, 2), (5, 7), (1, 1)])
def test_chunk_lists(num, chunk):
    got = ref_chunks(1, num, chunk)
    assert sum(n for _, n in got) == num
    assert [c for c, _ in got] == sorted(c for c, _ in got)
    # chunks larger than the range solve it in one remainder chunk
    if chunk >= num:
        assert got == [(1, num)]


def step_states(cfg_kw, n=16, steps=2, seed=3):
    cfg = W.lmea_config(n, **TIGHT, **cfg_kw)
    o = Oracle(cfg)
    o.set_state(0, W.lmea_state(cfg, seed))
    st = o.step(steps)
    return o.get_state(), st


def test_oracle_multicomp_step_matches_plain_step():
    plain, sp = step_states({})
    for kw in (dict(multicompsolves=1), dict(multicompsolves=1, comp_ion_chunks=2),
               dict(multicompsolves=1, comp_ion_chunks=1, comp_neutral_chunks=1)):
        mc, sm = step_states(kw)
        for c in range(8):
            assert rel(mc[c], plain[c]) <= 1e-12, (kw, c)
    # one solve per chunk: electrons, energy, one ion chunk, one neutral
    # chunk (the background species included) per step, one V-cycle each
    _, sm = step_states(dict(multicompsolves=1))
    assert sm.species_iterations == 2 * 4


def test_oracle_robin_wall_forces_single_component_chunks():
    # a Robin ion wall on the low x side: the ions go one by one, so the
    # step equals the plain one bit for bit
    kw = dict(multicompsolves=1)
    cfg = W.lmea_config(12, **TIGHT, **kw)
    cfg["ion_bc_lo"] = [4, 2, 2]
    o = Oracle(cfg)
    o.set_state(0, W.lmea_state(cfg, 4))
    st = o.step(1)
    # electrons + energy + 5 single ions + the neutral chunk of 2
    assert st.species_iterations == 8


def diffusion_case(n=16, dt=1.0, **kw):
    """The LMEA ions at a step where diffusion dominates (D dt / dx^2 ~ 3),
    so that the chunk's solve needs several V-cycles and a real bottom
    solve."""
    cfg = W.lmea_config(n, dt=dt, **kw)
    S = W.lmea_state(cfg, 5)
    o = Oracle(cfg)
    o.set_state(0, S)
    o.solve_potential(0.0)
    S = o.get_state()
    o.close()
    return cfg, S, np.zeros((9,) + S.shape[1:])


def test_oracle_joint_solve_matches_separate_solves():
    cfg, S, ex = diffusion_case(**TIGHT)
    o = Oracle(cfg)
    o.set_state(0, S)
    st = o.implicit_solve_chunk(1, 5, ex)
    assert st.converged and st.iterations >= 4
    joint = o.get_state(1, 5)
    for q, sp in enumerate(range(1, 6)):
        o.set_state(0, S)
        o.implicit_solve_scalar(sp, ex)
        assert rel(o.get_state(sp, 1)[0], joint[q]) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 24])
def test_joint_solve_parity(require_gpu, n):
    cfg, S, ex = diffusion_case(n=n, **TIGHT)
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    g.set_state(0, S)
    o.set_state(0, S)
    sg = g.implicit_solve_chunk(1, 5, ex)
    so = o.implicit_solve_chunk(1, 5, ex)
    assert sg.converged and so.converged
    assert abs(sg.iterations - so.iterations) <= 1
    Jg, Jo = g.get_state(1, 5), o.get_state(1, 5)
    for q in range(5):
        assert rel(Jg[q], Jo[q]) < 1e-12, (q, rel(Jg[q], Jo[q]))
    # the neutral pair, background species included (written, as the
    # reference's implicit_solve_scalar writes every species of its chunk).
    # The joint stopping norm is the background gas's, ten orders of
    # magnitude above the transported neutral, so the neutral stops at a
    # looser tolerance of its own: 1e-11 here
    g.set_state(0, S)
    o.set_state(0, S)
    g.implicit_solve_chunk(6, 2, ex)
    o.implicit_solve_chunk(6, 2, ex)
    for q, sp in enumerate((6, 7)):
        assert rel(g.get_state(sp, 1), o.get_state(sp, 1)) < 1e-11, sp


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(multicompsolves=1),
                                dict(multicompsolves=1, comp_ion_chunks=2),
                                dict(multicompsolves=1, do_bg_reactions=1,
                                     num_timestep_correctors=2)])
def test_multicomp_step_parity(require_gpu, kw):
    cfg = W.lmea_config(24, **TIGHT, **kw)
    S0 = W.lmea_state(cfg, 9)
    g, o = vb.Vidyut(cfg), Oracle(cfg)
    g.set_state(0, S0)
    o.set_state(0, S0)
    for s in range(2):
        g.step(1)
        o.step(1)
        Sg, So = g.get_state(), o.get_state()
        for c in list(range(8)) + [g.info["een_id"], g.info["pot_id"]]:
            r = rel(Sg[c], So[c])
            assert r < 1e-11, (s, c, r)
    if kw.get("do_bg_reactions"):
        assert rel(Sg[6], S0[6]) > 1e-14   # the background species reacted
