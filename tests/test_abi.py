"""The C ABI library loads on a machine without a GPU and exports every entry point that
include/*.h declares; host-side logic that needs no device is exercised directly."""

import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names += re.findall(r"^CKG_API\s+[\w\s\*]+?\b(ckg_\w+)\s*\(", src, flags=re.M)
    return names


def test_every_declared_symbol_is_exported(ckg):
    lib = ckg.lib()
    names = declared_functions()
    assert len(names) >= 50
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_codes_and_messages(ckg):
    """Argument errors come back as status codes with a message, not as crashes."""
    with __import__("pytest").raises(ckg.InvalidParams):
        ckg.primes_for_bits(16, [61], [60])
    assert ckg.lib().ckg_abi_version() == 1


def test_primes_for_bits_match_oracle(ckg, oracle):
    for log_n, qb, pb in [(13, [45] * 4, [60]), (16, [50] * 24, [60] * 8), (12, [60, 40, 40, 40, 40, 40], [60, 60])]:
        P = oracle.Params.from_bits(log_n, qb, pb, 40, 1)
        assert ckg.primes_for_bits(log_n, qb, pb) == (P.q, P.p)


def test_product_does_not_touch_the_oracle():
    """The product (package, C++/CUDA sources) never loads or names the oracle."""
    pkg = os.path.join(ROOT, "ckks-train_b200")
    for path in glob.glob(os.path.join(pkg, "**", "*"), recursive=True):
        if os.path.isfile(path) and path.endswith((".py", ".cu", ".cuh", ".hpp", ".cpp", ".h")):
            text = open(path).read()
            assert "oracle" not in text.lower(), path
