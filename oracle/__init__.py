"""ORACLE -- test infrastructure only.

CPU statements of the reference's algorithm for the compressed state-vector
path, used as the checker by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py.  Nothing in the product imports this package.

* csim_ref   -- the reference's own FP64 kernels (Qulacs csim, compiled from
                the reference sources by oracle/Makefile into _ref/).
* planner    -- partition_circuit / make_block_groups /
                build_stage_group_execution_plan restated in Python.
* pipeline   -- the CPU group loop (process_SV_group and the block-pair gate
                loops) restated over numpy blocks, with a pluggable codec.
* codec      -- the block codec's C statement (codec_oracle.c) and an
                emulation of the reference's compander + Bitcomp quantiser.
"""
