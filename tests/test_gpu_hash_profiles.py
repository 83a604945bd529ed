"""GPU proofs in the sha3-384 and sha3-512 hash profiles (separate library builds,
selected per process with STARK_GPU_HASH): Merkle roots, STIR and classic
DEEP-FRI proofs (n0 = 2^3 .. 2^16) and SHA-256 binding proofs byte-identical to
the oracle's build of the same profile, and accepted by the library's verifier."""
import os
import subprocess

import pytest

from test_hash_profiles_cpu import ROOT, run_checks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    # the profile builds are separate libraries: rebuild them if a source changed
    subprocess.run(["make", "-s", "-j3", "-C", os.path.join(ROOT, "oracle"), "all"], check=True)
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "stark-swarm_b200"), "profiles"], check=True)


@pytest.mark.parametrize("profile", ["sha3-384", "sha3-512"])
def test_gpu_profile_matches_oracle(profile):
    assert "ok" in run_checks(profile, "gpu", timeout=900)
