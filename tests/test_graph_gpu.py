"""CUDA-graph capture and replay of partition calls (mdx_graph_*): the
captured call is replayed after the input's contents change in place, and
every replay must equal the oracle on the current contents."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_plain_partition_graph_replays(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    n, m = 1_000_003, 8
    d = torch.empty(n, dtype=torch.int32, device="cuda")
    out = torch.empty_like(d)
    sizes = torch.empty(m, dtype=torch.uint32, device="cuda")
    flags = torch.empty(n, dtype=torch.uint32, device="cuda")
    g = mdx.capture_partition(d, ("mod", m), out, sizes, flags)
    for seed in (1, 2, 3):
        x = oracle.fill_uniform_u32(n, seed)
        d.copy_(torch.from_numpy(x.view(np.int32)))
        g.launch()
        torch.cuda.synchronize()
        eo, es, ef = oracle.partition(x, m, headflags=True)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), eo)
        assert np.array_equal(sizes.cpu().numpy(), es)
        assert np.array_equal(flags.cpu().numpy(), ef)
    g.close()


def test_segmented_graph_replays(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    rng = np.random.default_rng(8)
    lengths = np.clip(np.rint(rng.lognormal(np.log(1024), 1.5, size=3000)), 1, 1 << 22).astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.uint64)
    n, m = int(offs[-1]), 4
    d = torch.empty(n, dtype=torch.int32, device="cuda")
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    out = torch.empty_like(d)
    seg_sizes = torch.empty((len(lengths), m), dtype=torch.uint32, device="cuda")
    g = mdx.capture_partition_segmented(d, do, ("mod", m), out, seg_sizes)
    for seed in (5, 6):
        x = oracle.fill_uniform_u32(n, seed)
        d.copy_(torch.from_numpy(x.view(np.int32)))
        g.launch()
        torch.cuda.synchronize()
        eo, es = oracle.partition_segmented(x, offs, m)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), eo)
        assert np.array_equal(seg_sizes.cpu().numpy(), es)
    g.close()
