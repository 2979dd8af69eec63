"""Shared test helpers: building sums from Pauli strings and comparing term maps."""

from __future__ import annotations

import numpy as np

from ppvm_b200 import gates as G
from oracle.pyoracle import OracleSum


def planes(words, n):
    W = G.words(n)
    x = np.zeros((len(words), W), dtype=np.uint64)
    z = np.zeros((len(words), W), dtype=np.uint64)
    for i, s in enumerate(words):
        x[i], z[i] = G.parse_word(s, n)
    return x, z


def oracle_from(terms, n, thr=1e-10, maxw=None, clifford_angles=False):
    s = OracleSum(n, thr, maxw, clifford_angles)
    if terms:
        x, z = planes([t for t, _ in terms], n)
        s.add_terms(x, z, np.array([c for _, c in terms], dtype=np.float64))
    return s


def lossy_planes(words, n):
    W = G.lossy_words(n)
    x = np.zeros((len(words), W), dtype=np.uint64)
    z = np.zeros((len(words), W), dtype=np.uint64)
    for i, s in enumerate(words):
        x[i], z[i] = G.parse_lossy_word(s, n)
    return x, z


def lossy_oracle_from(terms, n, thr=0.0, maxw=None, max_loss_weight=None, clifford_angles=False):
    """An oracle sum of LossyPauliWord terms ('L' marks a lost qubit)."""
    s = OracleSum(n, thr, maxw, clifford_angles, lossy=True, max_loss_weight=max_loss_weight)
    if terms:
        x, z = lossy_planes([t for t, _ in terms], n)
        s.add_terms(x, z, np.array([c for _, c in terms], dtype=np.float64))
    return s


def lossy_dict(s):
    x, z, c = s.export()
    return {G.lossy_word_str(x[i], z[i], s.n): float(c[i]) for i in range(len(c))}


def lossy_list(s):
    x, z, c = s.export()
    return [(G.lossy_word_str(x[i], z[i], s.n), float(c[i])) for i in range(len(c))]


def term_dict(x, z, c, n):
    return {G.word_str(x[i], z[i], n): float(c[i]) for i in range(len(c))}


def oracle_dict(s):
    x, z, c = s.export()
    return term_dict(x, z, c, s.n)


def oracle_list(s):
    x, z, c = s.export()
    return [(G.word_str(x[i], z[i], s.n), float(c[i])) for i in range(len(c))]
