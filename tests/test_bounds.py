"""The opt-in bounds checker's registry (include/ckg.h, ckg_debug_bounds), on the CPU: a range
inside a live allocation passes, one that runs past its end or starts in freed memory fails with
the device status and a message naming it, unknown memory passes, and a new allocation over a
freed range is live again. The launch-side checks use the same registry."""

import pytest

BASE = 1 << 40  # synthetic addresses: the registry only compares them


@pytest.fixture()
def bounds(ckg):
    L = ckg.lib()

    def call(op, p=0, n=0):
        return L.ckg_debug_bounds(op, p, n)

    assert call(0, 0, 1) == 0  # on
    yield call, ckg
    call(0, 0, 0)  # off


def test_ranges(bounds):
    call, ckg = bounds
    call(1, BASE, 4096)
    assert call(3, BASE, 4096) == 0
    assert call(3, BASE + 1024, 1024) == 0
    assert call(3, BASE + 4096 - 8, 8) == 0
    assert call(3, BASE + 4096 - 8, 16) == ckg.Device.code
    assert "runs past its allocation" in ckg.lib().ckg_last_error().decode()
    assert call(3, BASE + (1 << 30), 1 << 20) == 0  # memory the library did not allocate
    call(2, BASE)
    assert call(3, BASE + 512, 8) == ckg.Device.code
    assert "freed memory" in ckg.lib().ckg_last_error().decode()
    call(1, BASE, 2048)  # reallocated: live again, with its new size
    assert call(3, BASE + 512, 8) == 0
    assert call(3, BASE + 1024, 2048) == ckg.Device.code
    call(2, BASE)


def test_off_checks_nothing(bounds):
    call, ckg = bounds
    call(1, BASE + (1 << 32), 64)
    call(0, 0, 0)
    assert call(3, BASE + (1 << 32), 1 << 20) == 0
    call(0, 0, 1)
    assert call(3, BASE + (1 << 32), 1 << 20) == ckg.Device.code
    call(2, BASE + (1 << 32))


def test_python_switch(bounds):
    call, ckg = bounds
    call(1, BASE + (1 << 34), 64)
    ckg.set_bounds_checking(False)
    assert call(3, BASE + (1 << 34), 128) == 0
    ckg.set_bounds_checking(True)
    assert call(3, BASE + (1 << 34), 128) == ckg.Device.code
    call(2, BASE + (1 << 34))
