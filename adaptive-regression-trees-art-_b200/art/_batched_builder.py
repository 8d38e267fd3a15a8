"""FIFO level/cohort scheduling (reference art/_batched_builder.py:20-62).

``build_bfs`` pops at most ``node_batch_size`` jobs, prepares them (top-up,
fit, stopping rules) and hands the ready ones to ``split_batch`` -- one
device launch sequence per cohort with the level dispatcher -- then
attaches the returned nodes in input order and enqueues their children
(left, then right).
"""

from __future__ import annotations

from collections import deque
from typing import TYPE_CHECKING, Callable

from .tree import SplitNode, TreeNode

if TYPE_CHECKING:
    from .builder import RegressionTreeBuilder, _NodeWork


def build_bfs(builder: "RegressionTreeBuilder", work: "_NodeWork",
              split_batch: Callable[[list], list[TreeNode]] | None = None) -> TreeNode:
    queue = deque([work])
    root = None

    def attach(job, node):
        nonlocal root
        if job.parent is None:
            root = node
        else:
            setattr(job.parent, job.side, node)

    while queue:
        ready = []
        # children about to be prepared get their samples in one launch, with
        # the builder's draws taken in the same order as one at a time
        cohort = [queue[i] for i in range(min(len(queue), builder.node_batch_size))]
        builder._top_up_cohort(cohort)
        # and their node models in one batched solve
        builder._fit_cohort(cohort)
        while queue and len(ready) < builder.node_batch_size:
            job = queue.popleft()
            leaf = builder._prepare_node(job)
            if leaf is None:
                ready.append(job)
            else:
                attach(job, leaf)
        if not ready:
            continue
        nodes = [builder._split_node(j) for j in ready] if split_batch is None else split_batch(ready)
        if len(nodes) != len(ready):
            raise RuntimeError("Split dispatch must return one node per ready job.")
        for job, node in zip(ready, nodes):
            attach(job, node)
            if isinstance(node, SplitNode):
                queue.extend(builder._children(job, node))
    assert root is not None
    return root
