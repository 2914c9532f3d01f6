"""Source rules of the CUDA code, checked as text (no device needed).

A warp collective (__shfl*_sync, __ballot_sync, __all_sync, __any_sync,
__match*_sync, __reduce*_sync) with the full mask must be reached by all 32
lanes.  Placed after `||`, `&&` or `?` in one statement, it is skipped by the
lanes whose earlier operand already decides the expression, and the other
lanes wait on them.  The collective's own arguments may hold such operators:
they are evaluated by every lane before the call."""
import glob
import os
import re

from conftest import ROOT

CSRC = os.path.join(ROOT, "pyquante_b200", "csrc")
COLLECTIVE = re.compile(r"__(shfl(_up|_down|_xor)?|ballot|all|any|match_any|match_all|reduce_[a-z]+)_sync\s*\(")
SHORT_CIRCUIT = re.compile(r"\|\||&&|\?")


def _strip(src):
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    src = re.sub(r"//[^\n]*", " ", src)
    return re.sub(r'"(\\.|[^"\\])*"', '""', src)


def _statements(src):
    """Text between statement boundaries (; { }), with the line of its end."""
    start, line = 0, 1
    for i, ch in enumerate(src):
        if ch == "\n":
            line += 1
        if ch in ";{}":
            yield src[start:i], line
            start = i + 1


def _guarded_collectives(stmt):
    """Collective calls that a ||, && or ?: earlier in the statement may skip
    (text inside an earlier collective's own argument list does not count)."""
    out = []
    for m in COLLECTIVE.finditer(stmt):
        # the text before this call, without the argument lists of earlier
        # collectives (up to one level of nested parentheses)
        head = re.sub(r"__\w+_sync\s*\([^()]*(\([^()]*\)[^()]*)*\)", "", stmt[:m.start()])
        if SHORT_CIRCUIT.search(head):
            out.append(m.group(0))
    return out


def test_no_warp_collective_behind_a_short_circuit():
    bad = []
    for path in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh"))):
        src = _strip(open(path).read())
        for stmt, line in _statements(src):
            for call in _guarded_collectives(stmt):
                bad.append("%s:%d: %s" % (os.path.basename(path), line, call))
    assert not bad, "warp collectives that some lanes may skip:\n" + "\n".join(bad)


def test_the_rule_catches_both_known_shapes():
    assert _guarded_collectives("const bool last = lane == 31 || __shfl_down_sync(0xffffffffu, k, 1) != k")
    assert _guarded_collectives("bool ok = a && __all_sync(0xffffffffu, b)")
    assert _guarded_collectives("x = c ? __shfl_sync(0xffffffffu, v, 0) : 0")
    assert not _guarded_collectives("if (__all_sync(0xffffffffu, skip || !live)) continue")
    assert not _guarded_collectives("const long long kn = __shfl_down_sync(0xffffffffu, key, 1)")
    assert not _guarded_collectives("v += __shfl_xor_sync(0xffffffffu, v, o)")
