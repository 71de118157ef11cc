"""Large device blocks (above 128 MB) that a freed interaction leaves are kept
for the next one, and rad.UtiDelAll returns them to the driver."""
import pytest

import models as MD


@pytest.mark.gpu
def test_utidelall_returns_kept_blocks_to_the_driver(rad, cuda):
    import torch

    h = MD.hybrid_undulator(rad)[0]  # about 6,000 elements: an 18,240^2 FP64 matrix of 2.7 GB
    im = rad.RlxPre(h, storage="f64")
    torch.cuda.synchronize()
    free_held, _ = torch.cuda.mem_get_info()
    rad.UtiDel(im)
    free_kept, _ = torch.cuda.mem_get_info()
    # the matrix block stays with the library after the interaction is freed
    assert abs(free_kept - free_held) < (256 << 20)
    im = rad.RlxPre(h, storage="f64")
    torch.cuda.synchronize()
    free_reused, _ = torch.cuda.mem_get_info()
    assert abs(free_reused - free_held) < (256 << 20)
    rad.UtiDelAll()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after - free_held >= 2 << 30


_EVICT = r"""
import os, sys
sys.path[:0] = [os.path.join(%(root)r), os.path.join(%(root)r, "tests")]
import torch
import models as MD
from radiacuda_b200 import rad
torch.cuda.init()
hX = MD.hybrid_undulator(rad)[0]                 # 6,080 elements: 2.66 GB FP64 matrix
im = rad.RlxPre(hX, storage="f64")
torch.cuda.synchronize()
rad.UtiDel(im)
f1, _ = torch.cuda.mem_get_info()                 # the 2.66 GB block is cached
hY = MD.hybrid_undulator(rad, n_pairs=60)[0]      # 4,560 elements: 1.50 GB
im = rad.RlxPre(hY, storage="f64")
torch.cuda.synchronize()
rad.UtiDel(im)
f2, _ = torch.cuda.mem_get_info()                 # 1.50 GB cached; 2.66 + 1.50 > the cap
print("DELTA", f2 - f1)
"""


@pytest.mark.gpu
def test_a_full_cache_keeps_the_newest_block(cuda):
    """With the cache capped at 3.5 GB, releasing a 1.50 GB matrix after a
    2.66 GB one displaces the older block instead of dropping the new one:
    free device memory grows by about the difference."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, RADB200_BUFCACHE_GB="3.5")
    r = subprocess.run([sys.executable, "-c", _EVICT % {"root": root}], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    delta = int([ln for ln in r.stdout.splitlines() if ln.startswith("DELTA")][0].split()[1])
    assert delta > 0.9e9, delta
