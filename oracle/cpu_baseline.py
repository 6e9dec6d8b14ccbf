"""Timed CPU restatement of the FLCF search (the CPU baseline).

TEST/BASELINE INFRASTRUCTURE ONLY: bench.py's CPU-baseline leg and the
reference arm import this; the product never does.

The reference's own path (MATLAB + MEX) cannot run here: MATLAB, Octave and
FFTW are absent.  This is its reference-precision restatement:
* rotation: the reference's compiled rot3d (oracle/_ref/libref_rotate.so)
  when built, else the oracle's bit-identical C restatement;
* FFTs: scipy.fft rfftn/irfftn in FP32 with all host threads (pocketfft in
  place of MATLAB's FFTW-backed fftn);
* FLCF and max/arg-max in numpy FP32 in tom_os3_findTemplate order
  (search/tom_os3_corr.m:151-176, search/tom_os3_bestPeak.m:42-47).
"""
from __future__ import annotations

import os
import time

import numpy as np
import scipy.fft as sfft

import tm_oracle as O


class CpuFLCF:
    def __init__(self, volume, template, mask, workers=None):
        self.workers = workers or os.cpu_count()
        self.N = tuple(volume.shape)
        t, self.tmean, self.tstd = O.prepare_template(template, mask)
        self.t = t.astype(np.float32)
        self.mask = np.asarray(mask, np.float32)
        mean, std, M = O.local_stats(volume, mask)
        self.mean = mean.astype(np.float32)
        self.std = std.astype(np.float32)
        self.M = np.float32(M)
        self.fimage = sfft.rfftn(np.asarray(volume, np.float32), workers=self.workers)
        self.den = (np.float32(self.tstd) * self.std).astype(np.float32)
        self.ccc = np.full(self.N, -1000, np.float32)
        self.idx = np.full(self.N, -1, np.int32)
        self.use_ref = O.ref_available()

    def rotate(self, e):
        if self.use_ref:
            return O.ref_rotate(self.t, e)
        return O.rotate(self.t, e)

    def step(self, e, index):
        t = self.rotate(e) * self.mask
        p = np.zeros(self.N, np.float32)
        T = t.shape
        o = [n // 2 - s // 2 for n, s in zip(self.N, T)]
        p[o[0]:o[0] + T[0], o[1]:o[1] + T[1], o[2]:o[2] + T[2]] = t * self.mask
        ft = sfft.rfftn(p, workers=self.workers)
        num = sfft.irfftn(self.fimage * np.conj(ft), s=self.N, workers=self.workers)
        num = np.fft.ifftshift(num) / self.M - self.mean * np.float32(self.tmean)
        cc = np.where(self.den != 0, num / np.where(self.den != 0, self.den, 1), 0).astype(np.float32)
        upd = self.ccc < cc
        self.ccc[upd] = cc[upd]
        self.idx[upd] = index

    def run(self, eulers, index0=0):
        t0 = time.perf_counter()
        for r, e in enumerate(np.asarray(eulers).reshape(-1, 3)):
            self.step(e, index0 + r)
        return time.perf_counter() - t0
