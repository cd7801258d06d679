"""A rank process for tests/test_replicas.py: joins the gloo group from the launcher's
environment (RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT), takes the maximum of (rank + 1) over
the ranks as bench.py takes its job time, and rank 0 prints the result as one JSON line."""
import datetime
import json
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'mpas-sw-tl-ad_b200'))

import torch.distributed as dist  # noqa: E402

from mpsw import replicas  # noqa: E402

dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=60))
rank, world = replicas.rank_world()
top = replicas.max_over_ranks(rank + 1.0)
if rank == 0:
    print(json.dumps({'world': world, 'max': top, 'local_rank': int(os.environ['LOCAL_RANK'])}), flush=True)
dist.barrier()
dist.destroy_process_group()
