"""Committed golden states (tests/golden/states.json, made by
tests/golden/make_golden.py from the CPU oracle): small seeded systems of
every feature mix, stepped to the end, reduced to counts and SHA-256 digests
of their IEEE bytes.  The oracle must reproduce them (CPU test) and so must
the CUDA path (GPU test), bit for bit.  The registry case registers a column
of every AtomData flag class (forward width 3, reverse width 2, zero, and an
unflagged width-2 column that is only permuted and copied to ghosts), written
by a test consumer: the oracle's column probe, and on the GPU
tests/hooks/registry_hook.cu through the force-hook ABI."""
import json
import os
import sys

import pytest

import oracle
from helpers import attach_oracle_probe, attach_registry_hook, build_hook
from soil_b200 import system

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import CASES, build, state_digest  # noqa: E402

with open(os.path.join(HERE, "golden", "states.json")) as f:
    GOLDEN = json.load(f)


def test_fixture_covers_every_case():
    assert sorted(GOLDEN) == sorted(CASES)


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden_state(name):
    s, steps = build(oracle.OracleSystem, name, attach=attach_oracle_probe)
    s.step(steps)
    assert state_digest(s) == GOLDEN[name]


@pytest.fixture(scope="module")
def registry_lib(tmp_path_factory):
    return build_hook(tmp_path_factory.mktemp("hook"), "registry_hook")


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_reproduces_golden_state(ctx, registry_lib, name):
    s, steps = build(lambda b, c, dt: system.System(ctx, b, c, dt), name,
                     attach=attach_registry_hook(registry_lib, 1e3))
    s.step(steps // 3)  # in two calls: the deferred final half-kick is flushed between them
    s.step(steps - steps // 3)
    got = state_digest(s)
    s.close()
    assert got == GOLDEN[name]
