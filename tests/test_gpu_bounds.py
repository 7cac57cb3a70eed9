"""The bounds-checked build (liborbx_checked.so, -DORBX_BOUNDS_CHECK) on the
GPU.  In it every global access of the pyramid, detect, NMS and describe
stages and of the popcount matcher is tested against its buffer's extent; an
access outside is skipped and reported instead of made.  On the pair (odd
sizes, padded pitches, binding caps, 4K, WTA 3/4, patch 25, FAST score, the
persistent pair form), the batched forms, the host-buffer path and ragged k = 2
lists it must report nothing and give exactly the normal build's outputs.  A
second run plants the mistake in the checked extent, not in memory: the image
extent, as checked, ends two rows early, and the reads of those rows (memory
the test owns) must be reported."""
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import bounds_cases  # noqa: E402
import orbx  # noqa: E402
import synth  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "cuda-orb_b200", "liborbx_checked.so")


@pytest.fixture(scope="module")
def checked_run(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(CHECKED):
        pytest.fail("liborbx_checked.so not built (python cuda-orb_b200/build.py --checked)")
    out = str(tmp_path_factory.mktemp("bounds") / "checked.npz")
    env = dict(os.environ, ORBX_CHECKED="1")
    subprocess.run([sys.executable, os.path.join(ROOT, "tests", "bounds_cases.py"), out], env=env, check=True,
                   timeout=900)
    return dict(np.load(out))


def test_normal_build_has_no_record():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    assert not orbx.CHECKED and orbx.lib().orbx_bounds_checked() == 0
    ctx = orbx.Context(0, orbx.make_params())
    with pytest.raises(orbx.OrbxError) as e:
        ctx.bounds_report()
    assert e.value.status == orbx.ORBX_ERR_STATE
    ctx.close()


def test_checked_build_reports_nothing(checked_run):
    recs = {k: v for k, v in checked_run.items() if k.endswith(".bounds") and not k.startswith("slack")}
    assert len(recs) >= 17
    bad = {k: v.tolist() for k, v in recs.items() if v[0] != 0}
    assert not bad, bad


def test_checked_build_equals_normal_build(checked_run):
    want = bounds_cases.run(orbx, synth, torch)
    assert len(want) >= 70
    for k, v in want.items():
        assert k in checked_run, k
        assert checked_run[k].shape == v.shape and np.array_equal(checked_run[k], v), k


def test_checked_build_reports_planted_extent(checked_run):
    n, site, off, extent = checked_run["slack.bounds"].tolist()
    a, _, _ = synth.make_pair(333, 257, seed=950)
    full = 257 * a.shape[1]
    assert n > 0
    assert site in (1, 2), site  # kSitePyrLoad, kSitePyrPadLoad
    assert extent == full - 2 * a.shape[1]
    assert extent <= off < full, (off, extent, full)
