"""Static checks of the 2D engine's launch configuration (no GPU needed): every
fused pass is launched with the dynamic shared memory its attribute allows, and
the largest pass fits one B200 CTA at the largest slice (1024 points)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "hawassi_c_b200", "csrc", "hw2d_engine.cu")
MAX_SMEM_PER_CTA = 227 * 1024   # sm_100 opt-in limit of dynamic shared memory per block


def padded(m):   # hw_fft.cuh: slices are swizzled in place, no pad slots
    return m


def test_every_pass_launches_with_its_attribute():
    s = open(SRC).read()
    attrs = dict(re.findall(r"cudaFuncSetAttribute\(hw2d::(\w+)<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, "
                            r"\(int\)smem_bytes<M>\((\d+)\)\)", s))
    launches = re.findall(r"hw2d::(\w+)<M><<<[^;]*?smem_bytes<M>\((\d+)\)", s)
    assert len(attrs) >= 28 and len(launches) == len(attrs)
    assert all(attrs.get(k) == v for k, v in launches), [(k, v, attrs.get(k)) for k, v in launches]


def test_largest_pass_fits_a_cta_at_1024_points():
    s = open(SRC).read()
    slices = max(int(v) for v in re.findall(r"smem_bytes<M>\((\d+)\)", s))
    assert slices * padded(1024) * 16 <= MAX_SMEM_PER_CTA
    src_fft = open(os.path.join(ROOT, "hawassi_c_b200", "csrc", "hw_fft.cuh")).read()
    assert "constexpr int padded(int m) { return m; }" in src_fft   # the size the bound above assumes
