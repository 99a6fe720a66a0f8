"""Test helper: executes a compiled fused program (mcg_compile) on the CPU.

Every basic-event word comes from the oracle's materialised node words, so
the emulation checks the program compiler (operand order, accumulator ops,
slot allocation and reuse, spills to global slots, tallies) against the
oracle without a GPU.  Test infrastructure only.
"""
from __future__ import annotations

import numpy as np

OP_HALT, OP_IN_BE, OP_BE_DEF, OP_BEGIN, OP_IN_SLOT, OP_IN_CONST, OP_END, OP_CONST_DEF, OP_TALLY = range(9)
NEG = 1 << 7
SLOT_GLOBAL = 1 << 23
NO_SLOT = 0xFFFFFF
ALL = np.uint64(0xFFFFFFFFFFFFFFFF)
AND, OR, ATLEAST, XOR, NOT, NAND, NOR, NULL = range(8)


def emulate(ops: np.ndarray, g, words: np.ndarray, n_tally: int, variable_thresholds: bool = False):
    """Returns (tally_values, ones): tally_values[i] is the word vector the
    program counted for tally i (last TALLY wins), ones[i] its popcount sum.
    With variable_thresholds the basic-event ops carry node ids in w2."""
    W = words.shape[1]
    by_counter = {}
    for e in range(g.n_be):
        by_counter[(int(g.be_pdag_idx[e]) + 1, int(g.be_event_idx[e]) + 1, int(g.be_threshold[e]) & 0xFFFFFFFF)] = e
    smem, glob = {}, {}
    acc = np.zeros(W, np.uint64)
    last = np.zeros(W, np.uint64)
    cnt = [np.zeros(W, np.uint64) for _ in range(8)]
    conn = kk = nbits = 0
    tally_vals = [None] * n_tally
    ones = np.zeros(n_tally, np.uint64)

    def load(ref):
        return glob[ref & (SLOT_GLOBAL - 1)] if ref & SLOT_GLOBAL else smem[ref]

    def store(ref, v):
        if ref == NO_SLOT:
            return
        if ref & SLOT_GLOBAL:
            glob[ref & (SLOT_GLOBAL - 1)] = v.copy()
        else:
            smem[ref] = v.copy()

    def be_value(op):
        if variable_thresholds:
            e = int(op[2])
            assert (int(g.be_pdag_idx[e]) + 1, int(g.be_event_idx[e]) + 1) == (int(op[1]), int(op[3]))
            return words[e]
        key = (int(op[1]), int(op[3]), int(op[2]))
        return words[by_counter[key]]

    for op in ops:
        code = int(op[0]) & 0xF
        if code == OP_HALT:
            break
        v = None
        if code in (OP_IN_BE, OP_BE_DEF):
            v = be_value(op)
        elif code == OP_IN_SLOT:
            v = load(int(op[1]))
        elif code in (OP_IN_CONST, OP_CONST_DEF):
            v = np.full(W, (int(op[2]) << 32) | int(op[1]), np.uint64)
        if code in (OP_IN_BE, OP_IN_SLOT, OP_IN_CONST):
            if int(op[0]) & NEG:
                v = ~v
            if conn in (AND, NAND):
                acc = acc & v
            elif conn in (OR, NOR):
                acc = acc | v
            elif conn == XOR:
                acc = acc ^ v
            elif conn == ATLEAST:
                carry = v
                for b in range(8):
                    if b < nbits:
                        t = cnt[b] & carry
                        cnt[b] = cnt[b] ^ carry
                        carry = t
            else:
                acc = v.copy()
        elif code in (OP_BE_DEF, OP_CONST_DEF):
            last = v
            store(int(op[0]) >> 8, last)
        elif code == OP_BEGIN:
            conn = (int(op[0]) >> 8) & 0xFF
            kk = (int(op[0]) >> 16) & 0xFF
            nbits = (int(op[0]) >> 24) & 0xF
            acc = np.full(W, ALL if conn in (AND, NAND) else 0, np.uint64)
            cnt = [np.zeros(W, np.uint64) for _ in range(8)]
        elif code == OP_END:
            if conn == ATLEAST:
                gt = np.zeros(W, np.uint64)
                eq = np.full(W, ALL, np.uint64)
                for b in range(7, -1, -1):
                    if (kk >> b) & 1:
                        eq = eq & cnt[b]
                    else:
                        gt = gt | (eq & cnt[b])
                        eq = eq & ~cnt[b]
                last = gt | eq
            elif conn in (NAND, NOR, NOT):
                last = ~acc
            else:
                last = acc.copy()
            store(int(op[1]), last)
        elif code == OP_TALLY:
            t = int(op[1])
            tally_vals[t] = last.copy()
            ones[t] += np.uint64(sum(bin(int(x)).count("1") for x in last))
        else:
            raise ValueError(f"unknown op {code}")
    return tally_vals, ones
