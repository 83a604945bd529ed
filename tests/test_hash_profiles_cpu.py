"""The sha3-384 and sha3-512 hash profiles (the reference's compile-time hash
features, hash/src/selected.rs:8-48) on the CPU. Each profile runs in a child
process with STARK_GPU_HASH set, since the oracle and the library are separate
builds per profile: the oracle's SHA3 against hashlib, its Merkle roots and the
packed-f0 root of its proofs against a hashlib restatement, STIR and classic
proofs that verify and reject flips, and the library's host verifier (the
profile's build) accepting those proofs and rejecting flips."""
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def run_checks(profile, mode, timeout=600):
    env = dict(os.environ, STARK_GPU_HASH=profile)
    r = subprocess.run([sys.executable, os.path.join(HERE, "hash_profile_checks.py"), mode], env=env,
                       capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


@pytest.fixture(scope="module", autouse=True)
def built():
    subprocess.run(["make", "-s", "-j3", "-C", os.path.join(ROOT, "oracle"), "all"], check=True)
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "stark-swarm_b200"), "profiles"], check=True)


@pytest.mark.parametrize("profile", ["sha3-384", "sha3-512"])
def test_oracle_profile(profile):
    assert "ok" in run_checks(profile, "oracle")


@pytest.mark.parametrize("profile", ["sha3-384", "sha3-512"])
def test_library_verifier_profile(profile):
    assert "ok" in run_checks(profile, "library")


def test_unknown_profile_is_refused():
    env = dict(os.environ, STARK_GPU_HASH="sha3-224")
    r = subprocess.run([sys.executable, "-c", f"import sys; sys.path.insert(0, {ROOT!r}); "
                        "import importlib; importlib.import_module('stark-swarm_b200')"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "STARK_GPU_HASH" in r.stderr
