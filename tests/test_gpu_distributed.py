"""The sharded grouped call (finoptions.distributed) on the CUDA engine, in a one-rank process group.

With one rank the shard is the whole batch, so the gathered result must equal the direct
price_lsm_call_grouped_batch call bit for bit; this runs the gather and result assembly around the
real engine (the two-rank sharding itself is covered on the CPU by test_distributed_sharding.py).
"""

from __future__ import annotations

import datetime
import socket

import numpy as np
import pytest
import torch.distributed as dist
from test_distributed_sharding import public_request

import finoptions as fo
from finoptions.distributed import price_lsm_call_grouped_batch_sharded

pytestmark = pytest.mark.gpu


def test_one_rank_sharded_call_equals_the_direct_call(executor) -> None:
    groups, mesh, method = public_request(states=12)
    direct = fo.price_lsm_call_grouped_batch(groups=groups, mesh=mesh, executor=executor, method=method)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sharded = price_lsm_call_grouped_batch_sharded(groups=groups, mesh=mesh, executor=executor, method=method)
    finally:
        dist.destroy_process_group()
    for name in ("prices", "sample_standard_deviations", "standard_errors", "regression_nodes",
                 "early_exercise_paths", "expiry_paths", "maximum_regression_condition_numbers"):
        np.testing.assert_array_equal(getattr(sharded, name), getattr(direct, name), err_msg=name)
    assert not sharded.prices.flags.writeable
