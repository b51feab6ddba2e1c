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
    # both kernels: the Gibbs array in tensor memory, 16 warps (the mixed kernel's shared-memory
    # form, both arrays there, would hold 11)
    assert E.use_tmem(53, False) and E.choose_block(53, False, True) == 512
    assert E.use_tmem(53, True) and E.choose_block(53, True, True) == 512
    assert E.choose_block(53, True) == 352
    # small mechanisms need no tensor memory to reach the block cap
    assert not E.use_tmem(10, False) and E.choose_block(10, False) == 512


def test_emitted_launch_shape_matches_the_choice():
    mech = synthetic.gri_shape()
    src = E.emit(mech)
    shapes = dict(re.findall(r"__launch_bounds__\((\d+), 1\) (cg_gen_\w+)\(", src)[i][::-1] for i in range(2))
    assert shapes == {"cg_gen_fp64": "512", "cg_gen_mixed": "512"}
    # one tensor-memory allocation per kernel, freed at its end; columns 2 ns per warp slot
    assert src.count("cgg::tm_alloc(&tm_slot, 512u)") == 2 and src.count("cgg::tm_free(tbase, 512u)") == 2
    assert "cgg::tm_thread_base(tbase, 106)" in src
    # every EGp load of a reaction stays inside the warp slot's columns
    offs = [int(x) for x in re.findall(r"tw \+ (\d+)u", src)]
    assert offs and max(offs) <= 2 * (mech.ns - 1)
    # barrier spacing per precision
    fp64, mixed = src.split("cg_gen_mixed(", 1)
    assert fp64.count("__syncthreads();") >= mech.nr // E.SYNC_EVERY
    assert mixed.count("__syncthreads();") >= mech.nr // E.SYNC_EVERY_MIXED


def test_fp64_values_of_three_reactions_share_one_wait():
    """FP64 kernel, tensor-memory mode: the values of EGP_GROUP consecutive
    reactions (in emission order) are issued together and completed by one
    wait whose operands are exactly those registers, and each reversible
    reaction reads only values of its own group."""
    mech = synthetic.gri_shape()
    order = E.reaction_order(mech)
    fp64 = E.emit(mech, precision="fp64")
    G = E.EGP_GROUP
    groups = [order[p:p + G] for p in range(0, len(order), G)]
    with_rev = [g for g in groups if any(mech.reactions[j].reversible for j in g)]
    waits = re.findall(r'asm volatile\("tcgen05\.wait::ld\.sync\.aligned;" : ([^:]*) :: "memory"\);', fp64)
    assert len(waits) == len(with_rev)
    for w, g in zip(waits, with_rev):
        sps = {sp for j in g if mech.reactions[j].reversible
               for sp in list(mech.reactions[j].reactants) + list(mech.reactions[j].products)}
        assert w.count('"+r"') == 2 * len(sps)
    assert "cgg::tm_ld(" not in fp64                # no per-reaction loads left
    # the per-reaction form is still available
    assert "cgg::tm_ld(" in E.emit(mech, precision="fp64", egp_group=1)


def test_tmem_option_for_the_mixed_kernel():
    mech = synthetic.synthetic_mechanism(20, 60, 4, 4, seed=91, name="synthetic_20_60_s91")
    src = E.emit(mech, tmem=True)
    assert src.count("cgg::tm_alloc") == 2
    mixed = src.split("cg_gen_mixed(", 1)[1]
    assert "sG[" not in mixed and "cgg::tm_ld(" in mixed


@pytest.mark.parametrize("factory", [synthetic.gri_shape, synthetic.h2o2_10sp, synthetic.all_kinds])
def test_live_range_order_is_a_permutation_that_shortens_live_ranges(factory):
    mech = factory()
    order = E.reaction_order(mech)
    assert sorted(order) == list(range(mech.nr))
    assert E.live_accumulators(mech, order) <= E.live_accumulators(mech, list(range(mech.nr)))
    if mech.ns == 53:
        assert E.live_accumulators(mech, order) <= 32


def test_each_wdot_is_stored_once_after_its_last_reaction():
    """Live-range mode: an accumulator is declared before the first reaction
    that touches its species and stored right after the last one; species no
    reaction touches are stored as zero; every species is stored once."""
    mech = synthetic.gri_shape()
    src = E.emit(mech, precision="fp64")
    body = src.split("cg_gen_fp64(", 1)[1].split("\n}\n", 1)[0]
    # outputs leave with streaming stores (evict-first), as the inputs arrive with streaming loads
    stores = re.findall(r"__stcs\(wdot \+ \(int64_t\)(\d+) \* ng \+ i, (w\d+|0\.0)\);", body)
    assert sorted(int(k) for k, _ in stores) == list(range(mech.ns))
    assert "wdot[" not in body and "Y[" not in body and body.count("__ldcs(Y + ") == mech.ns
    for k, v in stores:
        if v != "0.0":
            assert v == f"w{k}"
            decl = body.index(f" w{k} = 0.0")
            last_use = max(body.rfind(f"w{k} += "), body.rfind(f"w{k} -= "), body.rfind(f"w{k} = fma("))
            store = body.index(f"__stcs(wdot + (int64_t){k} * ng + i, w{k});")
            assert decl < last_use < store
    # the plain form is still available
    plain = E.emit(mech, precision="fp64", stream_io=False)
    assert "__stcs(" not in plain and f"wdot[(int64_t)0 * ng + i] = " in plain


@pytest.mark.slow
def test_generated_53_species_kernels_fit_their_register_budget(tmp_path):
    """ptxas's own register count and spills of the emitted 53-species
    kernels (nvcc cross-compiles; no GPU): each fits the registers its
    launch shape leaves per thread, with at most a few spilled words."""
    import subprocess
    from chemgen_b200.build import ARCH, FLAGS, nvcc
    mech = synthetic.gri_shape()
    src = tmp_path / "g.cu"
    src.write_text(E.emit(mech))
    r = subprocess.run([nvcc()] + ARCH + FLAGS + ["-I", E.os.path.join(E.HERE, "csrc"), "-Xptxas", "-v", "-c",
                        str(src), "-o", str(tmp_path / "g.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    info = {}
    for name, spill, regs in re.findall(r"Function properties for \w*?(cg_gen_\w+?)E.*?\n\s+\d+ bytes stack frame, "
                                        r"(\d+) bytes spill stores.*?\nptxas info\s+: Used (\d+) registers", r.stderr):
        info[name] = (int(regs), int(spill))
    shapes = {"cg_gen_fp64": E.choose_block(53, False, True), "cg_gen_mixed": E.choose_block(53, True)}
    assert set(info) == set(shapes), r.stderr[-2000:]
    for name, (regs, spill) in info.items():
        assert regs * shapes[name] <= E.REG_FILE, (name, regs)
        assert spill <= 64, (name, spill)
