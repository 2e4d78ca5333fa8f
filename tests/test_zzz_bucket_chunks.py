"""Grid buckets of a batch grow by chunks (jt_batch.cu, BucketChunk): boxes of
one grid size added after a first pass get a new chunk, the first pass's
grids stay in place, and a screened box's two slots may sit in different
chunks.  Forces against each box's single-box result."""
import numpy as np
import pytest

import janus_treepm as J
from test_gpu_batch import FORCE_TOL, _cmp, make_box

pytestmark = pytest.mark.gpu


def test_grid_bucket_grows_by_chunks():
    """Boxes of one grid size added after a first pass: the bucket grows by a
    chunk (the first pass's grids stay in place), and every box's forces
    still equal its own single-box result, with a screened box whose main
    slot is the first chunk's only one and whose unsigned source takes the
    first slot of the new chunk."""
    boxes = [(21, 12, 12, 64.0, 32, 19.0), (22, 10, 14, 60.0, 32, 7.0), (23, 12, 8, 70.0, 32, 11.0)]
    B = J.Batch()
    first = B.add(*make_box(*boxes[0]))
    B.forces([first])                       # bucket of 32^3 grids: one slot
    ids = [first] + [B.add(*make_box(*bx)) for bx in boxes[1:]]
    B.set_screening(ids[1], 5.0, 0.0)
    # slots in pass order: the screened box 0 (first chunk) and 1 (new
    # chunk), then 2 and 3: 4 slots, a chunk of 3 added
    B.forces([ids[1], ids[0], ids[2]])
    for k, (bid, box) in enumerate(zip(ids, boxes)):
        cfg, pp, vp, pm, vm = make_box(*box)
        s = J.Solver(cfg)
        if k == 1:
            s.set_screening(5.0, 0.0)
        s.set_state(pp, vp, pm, vm)
        rp, rm = s.accel()
        s.close()
        ap, am = B.accel(bid)
        _cmp(ap, rp.astype(np.float64), FORCE_TOL)
        _cmp(am, rm.astype(np.float64), FORCE_TOL)
    B.close()
