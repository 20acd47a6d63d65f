"""Tecplot output in the reference's binary layout (techead / strio /
write_output_file_mb, src/mo_io.f90:275-530), through the C ABI, on the CPU:
pinned against an independent numpy restatement of the header sequence."""
import numpy as np
import pytest

from canard_b200 import api


def i32(v):
    return np.int32(v).tobytes()


def strio(s):
    return b"".join(i32(ord(ch)) for ch in s) + i32(0)


def reference_bytes(n, arrays, time):
    """techead for block 0 (file header, every zone), then per block its zone
    section and its FP32 data."""
    mq = 3 if n == -1 else 5
    out = b"#!TDV112" + i32(1) + i32(min(n + 2, 2))
    out += strio("grid" if n == -1 else "n%03d" % n) + i32(mq)
    for name in (["x", "y", "z"] if n == -1 else ["rho", "u", "v", "w", "p"]):
        out += strio(name)
    for mm, a in enumerate(arrays):
        out += np.float32(299.0).tobytes() + strio("z%03d" % mm) + i32(-1) + i32(mm + 1)
        out += np.float64(time).tobytes() + i32(-1) + i32(0) + i32(0) + i32(0) + i32(0)
        out += i32(a.shape[3]) + i32(a.shape[2]) + i32(a.shape[1]) + i32(0)
    out += np.float32(357.0).tobytes()
    for a in arrays:
        out += np.float32(299.0).tobytes() + b"".join(i32(1) for _ in range(mq)) + i32(0) + i32(0) + i32(-1)
        for m in range(mq):
            out += np.float64(a[m].min()).tobytes() + np.float64(a[m].max()).tobytes()
        out += np.ascontiguousarray(a, np.float32).tobytes()
    return out


def blocks(mq, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((mq, 5, 4, 6)).astype(np.float32),
            rng.standard_normal((mq, 3, 7, 2)).astype(np.float32)]


def test_file_names():
    assert api.plt_name(-1) == "data/grid.plt"
    assert api.plt_name(0) == "data/n000.plt"
    assert api.plt_name(42) == "data/n042.plt"


@pytest.mark.parametrize("n", [-1, 0, 7])
def test_layout_matches_the_reference_sequence(tmp_path, n):
    arrays = blocks(3 if n == -1 else 5, n + 5)
    p = str(tmp_path / "out.plt")
    api.plt_write(p, n, arrays, time=0.0 if n == -1 else 1.25 + n)
    assert open(p, "rb").read() == reference_bytes(n, arrays, 0.0 if n == -1 else 1.25 + n)


def test_arguments_beyond_three_digit_names_are_rejected(tmp_path):
    with pytest.raises(api.CanardError) as e:
        api.plt_write(str(tmp_path / "x.plt"), 1000, blocks(5, 1))
    assert e.value.code == api.ERR_ARG
