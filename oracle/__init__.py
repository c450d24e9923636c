"""CPU oracle for the CVQPG fit iteration -- TEST INFRASTRUCTURE ONLY.

A restatement, in numpy float64 (and, for the timed CPU baseline, torch on the
host cores), of the reference algorithm of every stage of the hot path. Each
function cites the reference file:line it follows. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline leg and the
``--impl reference`` arm) may import this package, and only as the checker or
the CPU baseline; the product package never imports it.

Parity pinning: the splat, preprocessing, padding, loss control flow and Adan
restatements are pinned against fixtures generated by running the reference
itself (tests/golden/make_golden.py). The BLASM transfer function and the
defocus-target kernel (third-party ``odak`` 0.2.7) and SSIM (third-party
``pytorch_msssim`` 1.0.0) are not installed anywhere here: those restatements
follow the published algorithms and are "parity unpinned".
"""
