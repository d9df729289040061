"""Thread-local operation recording (restates jaqsi/tape.py:10-138).

Operations created inside ``with recording() as tape:`` are appended to
``tape`` by :class:`~jaqsi_b200.operations.Operation`; nesting pushes a fresh
tape per level, and each thread has its own stack.
"""
from __future__ import annotations

import threading
from contextlib import contextmanager
from typing import TYPE_CHECKING, Callable, Iterator, List, Optional

if TYPE_CHECKING:  # pragma: no cover
    from jaqsi_b200.operations import Operation

_local = threading.local()


def _tape_stack() -> List[List["Operation"]]:
    if not hasattr(_local, "stack"):
        _local.stack = []
    return _local.stack


def active_tape() -> Optional[List["Operation"]]:
    """The innermost recording tape of this thread, or ``None``."""
    stack = _tape_stack()
    return stack[-1] if stack else None


@contextmanager
def recording() -> Iterator[List["Operation"]]:
    """Record every operation created in the block onto a fresh tape."""
    stack = _tape_stack()
    tape: List["Operation"] = []
    stack.append(tape)
    try:
        yield tape
    finally:
        stack.pop()


def shift_and_append(tape_ops: List["Operation"], offset: int) -> None:
    """Append shallow copies of *tape_ops* with wires shifted by *offset*."""
    current = active_tape()
    if current is None:
        return
    for o in tape_ops:
        shifted = o.__class__.__new__(o.__class__)
        shifted.__dict__.update(o.__dict__)
        shifted._wires = [w + offset for w in o.wires]
        current.append(shifted)


def copy_to_tape(fn: Callable[[], None], offset: int) -> None:
    """Record *fn* on a side tape and replay it shifted by *offset*."""
    with recording() as side_tape:
        fn()
    shift_and_append(side_tape, offset)
