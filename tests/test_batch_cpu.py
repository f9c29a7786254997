"""Host logic of the batched blocks: seeded sizes, shelf packing with the
separating gap, particle counts, and the Gaussian random field."""
import numpy as np

from geowarp_b200 import batch


def test_sizes_are_seeded_and_in_range():
    a = batch.instance_sizes(64, seed=0)
    assert a == batch.instance_sizes(64, seed=0)
    assert all(32 <= nx <= 128 and 32 <= ny <= 64 for nx, ny in a)
    assert a != batch.instance_sizes(64, seed=1)


def test_shelf_pack_keeps_the_gap():
    sizes = batch.instance_sizes(64, seed=0)
    off, width, height = batch.shelf_pack(sizes)
    boxes = [(ox, oy, ox + nx, oy + ny) for (ox, oy), (nx, ny) in zip(off, sizes)]
    for (x0, y0, x1, y1) in boxes:
        assert x0 >= 0 and y0 >= 0 and x1 <= width and y1 <= height
    for i in range(len(boxes)):
        for j in range(i + 1, len(boxes)):
            a, b = boxes[i], boxes[j]
            dx = max(b[0] - a[2], a[0] - b[2])
            dy = max(b[1] - a[3], a[1] - b[3])
            assert max(dx, dy) >= batch.GAP, (a, b)
    # the packing is reasonably dense
    used = sum(nx * ny for nx, ny in sizes)
    assert used / (width * height) > 0.5


def test_random_field_statistics():
    f = batch.gaussian_random_field(96, 64, 2, 0.05, corr_len=0.5, std=0.3, seed=3)
    assert f.shape == (96 * 64 * 4,)
    assert abs(f.mean()) < 1e-12 and abs(f.std() - 0.3) < 1e-12
    # correlation at a lag of one correlation length along x: exp(-1) for the
    # Gaussian covariance, within sampling error of a field only a few lengths wide
    g = np.zeros((96 * 2, 64 * 2))
    i, j, px, py = np.meshgrid(np.arange(96), np.arange(64), np.arange(2), np.arange(2), indexing="ij")
    g[(i * 2 + px).ravel(), (j * 2 + py).ravel()] = f
    lag = int(round(0.5 / 0.025))
    c = np.mean(g[:-lag] * g[lag:]) / np.mean(g * g)
    assert 0.15 < c < 0.6, c
    # and the field is smooth: neighbours are strongly correlated
    c1 = np.mean(g[:-1] * g[1:]) / np.mean(g * g)
    assert c1 > 0.95
