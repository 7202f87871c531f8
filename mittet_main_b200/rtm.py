"""Residual re-injection (the time-reversed residual study of the reference).

corona/ver0030r_a drives the magnetic point sources of read_source_3d with a
recorded residual instead of the Gaussian derivative (read_source_3d_res,
corona/ver0030r_a/cpu_waveform.f90:62-85: Hz -= signal_res(istep) dt / myu /
(dx dy dz) at both source cells, before the E half step).  The residual is
the difference of a receiver trace between a model and its reference model
(py_residual_inout.py), reversed in time with the time axis kept
(py_rev_residual.py).  This module builds that signal and the wavelet array
the solver takes; the solve itself is the ordinary forward path.
"""
from __future__ import annotations

import numpy as np


def reversed_residual(trace: np.ndarray, reference_trace: np.ndarray) -> np.ndarray:
    """signal_res = (trace - reference_trace) reversed in time."""
    r = np.asarray(trace, dtype=np.float64) - np.asarray(reference_trace, dtype=np.float64)
    return np.ascontiguousarray(r[::-1])


def reinjection_wavelet(signal_res: np.ndarray) -> np.ndarray:
    """Wavelet array w[0..nt] for MittetSolver.set_wavelet: a magnetic point
    source takes w[istep] at step istep = 1..nt (signal_res(istep) of
    read_source_3d_res), so w = [0, signal_res(1), ..., signal_res(nt)]."""
    return np.concatenate([[0.0], np.asarray(signal_res, dtype=np.float64)])
