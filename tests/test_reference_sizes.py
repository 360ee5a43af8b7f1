"""The reference's CUDA build runs only at image sizes that are multiples of
16 in both directions: its accumulation kernels run 16x16 blocks with no
bounds guard, so any other size reads and writes past its layers. Host-side
checks of the two places that keep to this rule; no GPU is needed."""
import pytest

import bench
import oracle
from nectarrender_b200 import scenes


def test_bench_renders_the_reference_at_whole_blocks():
    spec = scenes.cornell(res=8, spp=2)
    spec.camera["resolution"] = (1080.0, 1920.0)
    padded, pixels = bench.padded_for_reference_cuda(spec)
    assert padded.camera["resolution"] == (1088.0, 1920.0)
    assert pixels == 1088 * 1920  # the rate counts the pixels rendered
    assert spec.camera["resolution"] == (1080.0, 1920.0)  # the caller's spec is untouched
    same, n = bench.padded_for_reference_cuda(scenes.cornell(res=64, spp=2))
    assert same.camera["resolution"] == (64.0, 64.0) and n == 64 * 64


@pytest.mark.parametrize("h,w", [(37, 48), (48, 37), (1080, 1920)])
def test_reference_cuda_refuses_partial_blocks(h, w):
    if not oracle.REF_CUDA_SO.exists():
        pytest.skip("reference CUDA build not present")
    spec = scenes.cornell(res=16, spp=2)
    spec.camera["resolution"] = (float(h), float(w))
    # refused on the host, before any CUDA call
    with pytest.raises(ValueError, match="multiple of 16"):
        oracle.RefCUDA().render(spec, 1, mode=0)
