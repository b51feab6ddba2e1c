"""Launch shape of the generated kernels (host logic, no GPU): the block
fills the shared-memory state and the register file, the Gibbs array moves
to tensor memory only when that lets the FP64 block grow, and every choice
stays within shared memory, the 512 tensor-memory columns and 1024 threads."""
import re

import pytest

from chemgen_b200 import emit_cuda as E
from chemgen_b200 import synthetic


@pytest.mark.parametrize("ns", range(1, E.MAX_REG_SPECIES + 1))
@pytest.mark.parametrize("mixed", [False, True])
def test_block_fits_every_resource(ns, mixed):
    tm = E.use_tmem(ns, mixed)
    b = E.choose_block(ns, mixed, tm)
    assert 32 <= b <= E.MAX_BLOCK and b % 32 == 0
    assert E.smem_per_species(mixed, tm, True) * ns * b <= E.SMEM_BUDGET
    if tm:
        assert -(-b // 128) * 2 * ns <= 512       # column slots of the warps sharing a lane quadrant
    regs = 2 * ns + (20 if tm else 64)
    assert b * regs <= E.REG_FILE or b == 32


def test_53_species_choices():
    # FP64: EGp in tensor memory, 16 warps; mixed: both arrays in shared memory, 11 warps
    assert E.use_tmem(53, False) and E.choose_block(53, False, True) == 512
    assert not E.use_tmem(53, True) and E.choose_block(53, True) == 352
    # small mechanisms need no tensor memory to reach the block cap
    assert not E.use_tmem(10, False) and E.choose_block(10, False) == 512


def test_emitted_launch_shape_matches_the_choice():
    mech = synthetic.gri_shape()
    src = E.emit(mech)
    shapes = dict(re.findall(r"__launch_bounds__\((\d+), 1\) (cg_gen_\w+)\(", src)[i][::-1] for i in range(2))
    assert shapes == {"cg_gen_fp64": "512", "cg_gen_mixed": "352"}
    # one tensor-memory allocation (FP64 kernel), freed at its end; columns 2 ns per warp slot
    assert src.count("cgg::tm_alloc(&tm_slot, 512u)") == 1 and src.count("cgg::tm_free(tbase, 512u)") == 1
    assert "cgg::tm_thread_base(tbase, 106)" in src
    # every EGp load of a reaction stays inside the warp slot's columns
    offs = [int(x) for x in re.findall(r"tw \+ (\d+)u", src)]
    assert offs and max(offs) <= 2 * (mech.ns - 1)
    # barrier spacing per precision
    fp64, mixed = src.split("cg_gen_mixed(", 1)
    assert fp64.count("__syncthreads();") >= mech.nr // E.SYNC_EVERY
    assert mixed.count("__syncthreads();") >= mech.nr // E.SYNC_EVERY_MIXED


def test_tmem_option_for_the_mixed_kernel():
    mech = synthetic.synthetic_mechanism(20, 60, 4, 4, seed=91, name="synthetic_20_60_s91")
    src = E.emit(mech, tmem=True)
    assert src.count("cgg::tm_alloc") == 2
    mixed = src.split("cg_gen_mixed(", 1)[1]
    assert "sG[" not in mixed and "cgg::tm_ld(" in mixed
