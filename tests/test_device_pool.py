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
