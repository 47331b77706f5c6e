"""The plain GPU form against the reference CPU core as it builds with the
stock C library, and a whole 16-frame 1080p YUV444PS clip.

The parity tests pin bit-exactness against the reference sources built with a
correctly rounded libm (oracle/libm_pin.c), so that every platform computes
the same bits.  The reference as users build it calls the stock glibc expf /
logf / log1pf / powf, whose last bits can differ.  The bar there is the one
stated for the plain form against the reference CPU path: at most 1e-4 max abs and 0.01 dB of
PSNR against the clean clip.  The second test runs the bench's workload
(1920x1080 YUV444PS, 16 frames, sigma 20, the CPU core's default parameters)
through Basic and Final on the GPU and compares every output frame with the
CPU core's, bit for bit.
"""
import os

import numpy as np
import pytest

import oracle as O
import synth
import vnlbcu

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-4   # the plain form's tolerance against the reference CPU path
MAX_DB = 0.01

CPU_DEFAULTS = dict(block_size=8, block_step=8, group_size=8, bm_range=9, radius=1, patch_time=1, rank=8,
                    cap_factor=4.0)
BASIC = dict(variance_threshold=1.1, weight_alpha=0.75, weight_beta=0.35, weight_gamma=1.0)
FINAL = dict(tau=400.0, variance_threshold=1.7, flat_areas=1, weight_alpha=1.0, weight_beta=0.5, weight_gamma=1.0)


def gpu_chain(noisy, sigma):
    basic = vnlbcu.Basic(noisy, sigma=sigma, **CPU_DEFAULTS, **BASIC)
    final = vnlbcu.Final(noisy, ref=basic, sigma=sigma, **CPU_DEFAULTS, **FINAL)
    return basic, final


def reference(kind, noisy, sigma):
    try:
        o = O.Oracle(kind)
    except FileNotFoundError:
        pytest.skip(f"the {kind} build of the reference core is absent (make -C oracle ref)")
    bp = O.cpu_params(O.BASIC, sigma, **CPU_DEFAULTS)
    fp = O.cpu_params(O.FINAL, sigma, **CPU_DEFAULTS)
    return o.chain(noisy, bp, fp, threads=os.cpu_count())


@pytest.mark.parametrize("w,h,frames,planes,sigma", [(256, 256, 8, 1, 10.0), (160, 128, 6, 3, 20.0)],
                         ids=["gray_256x256x8_sigma10", "yuv_160x128x6_sigma20"])
def test_plain_form_within_tolerance_of_the_stock_glibc_reference(w, h, frames, planes, sigma):
    clean, noisy = synth.make_clip(w, h, frames, planes, sigma, seed=0)
    gb, gf = gpu_chain(noisy, sigma)
    rb, rf = reference("ref_glibc", noisy, sigma)
    for name, g, r in (("basic", gb, rb), ("final", gf, rf)):
        assert float(np.max(np.abs(g - r))) <= MAX_ABS, name
        assert abs(synth.psnr(g, clean) - synth.psnr(r, clean)) <= MAX_DB, name


@pytest.mark.timeout(1200)
def test_sixteen_frames_1080p_yuv444_bit_exact():
    clean, noisy = synth.make_clip(1920, 1080, 16, 3, 20.0, seed=0)
    gb, gf = gpu_chain(noisy, 20.0)
    kind = "ref" if O.REF_LIB.exists() else "port"
    rb, rf = reference(kind, noisy, 20.0)
    for name, g, r in (("basic", gb, rb), ("final", gf, rf)):
        diff = np.flatnonzero(np.ascontiguousarray(g).view(np.uint32) != np.ascontiguousarray(r).view(np.uint32))
        assert diff.size == 0, (name, kind, diff.size, float(np.max(np.abs(g - r))))
    assert synth.psnr(gf, clean) > synth.psnr(noisy, clean)
