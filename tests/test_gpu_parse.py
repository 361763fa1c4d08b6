"""The batch decoder with its marker parse on the GPU (cjBatchSetParse(b, 1):
k_parse_headers, one thread per file) against the same batch parsed on the
host: the same error code for every file and byte-identical outputs, over
seeded encodes of every sampling mode and restart structure, the golden
fixtures (malformed files among them), progressive frames (rejected by the
batch decoder) and header mutations."""
import io

import numpy as np
import pytest
from PIL import Image

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def files(golden):
    out = [np.asarray(golden[k]["jpeg"], np.uint8).tobytes() for k in sorted(golden)]
    out += [s.data for s in W.mixed_batch(n=40, seed=71, max_side=700)]
    rng = np.random.default_rng(8)
    img = Image.fromarray(rng.integers(0, 255, (48, 80, 3), dtype=np.uint8))
    b = io.BytesIO()
    img.save(b, "JPEG", quality=80, progressive=True)
    out.append(b.getvalue())
    # header mutations of a few encodes
    for base in out[-8:-1]:
        sos = base.find(b"\xff\xda")
        for _ in range(4):
            m = bytearray(base)
            m[int(rng.integers(2, sos))] = int(rng.integers(0, 256))
            out.append(bytes(m))
    return out


def test_device_parse_equals_host_parse(cj, files):
    res = {}
    for on_device in (False, True):
        with cj.Batch() as b:
            b.set_parse(on_device)
            res[on_device] = b.decode(files)
    (img_h, err_h), (img_d, err_d) = res[False], res[True]
    assert err_h == err_d
    assert sum(1 for e in err_h if e) >= 5 and sum(1 for e in err_h if not e) >= 40
    for k, e in enumerate(err_h):
        if not e:
            assert np.array_equal(img_h[k], img_d[k]), k
