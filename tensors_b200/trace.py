"""Phase ranges of the library (NVTX ranges named with the reference's
TOOLS_PTIMER tags), recorded on the host for inspection without a profiler."""
from __future__ import annotations

import ctypes
from contextlib import contextmanager

from ._lib import lib


def record(enabled: bool = True) -> None:
    """Clear the host-side list of phase ranges and start (or stop) recording."""
    lib().tb_trace_record(1 if enabled else 0)


def names() -> list[str]:
    """The phase ranges entered since recording started, in order."""
    need = lib().tb_trace_names(None, 0)
    buf = ctypes.create_string_buffer(int(need))
    lib().tb_trace_names(buf, int(need))
    return [s for s in buf.value.decode().split("\n") if s]


def times() -> list[tuple[str, float]]:
    """(name, host wall milliseconds) of every phase range entered since recording started, in
    order (-1.0 for a range still open)."""
    got = names()
    n = int(lib().tb_trace_times(None, 0))
    ms = (ctypes.c_double * max(n, 1))()
    lib().tb_trace_times(ms, n)
    return list(zip(got, [float(ms[i]) for i in range(min(n, len(got)))]))


@contextmanager
def recording():
    """with recording() as got: ... ; got holds the ranges entered inside the block."""
    got: list[str] = []
    record(True)
    try:
        yield got
    finally:
        got.extend(names())
        record(False)
