"""The tensor-map layouts of the guide's training kernels, checked on the host.

The forward and backward store a slot's 128 x 64 bf16 operand tile with one TMA bulk tensor store
through a 5D map {8 features, 8 rows (stride 128 B), 8 chunks (stride 16 B), row groups (stride
1 KB), layers}; the weight-gradient kernel loads the 48-wide output gradient through a 3D map
{8 features, 32 records (stride 96 B), 6 groups (stride 16 B)}. A TMA box lands in (or is read
from) shared memory densely, innermost dimension first. These tests walk each box in that order
and check that element k of the box sits where the tcgen05 operand layout wants it in shared
memory and where the row-major tensor holds it in global memory (liar_b200/csrc/guide.cu:
ensure_tensor_maps, k_eval_tc, k_train_bwd_tc, k_train_dw_tc).
"""
import itertools

import numpy as np


def box_order(dims):
    """Coordinates of a box's elements in TMA order (the first dimension fastest)."""
    for idx in itertools.product(*[range(d) for d in reversed(dims)]):
        yield tuple(reversed(idx))


def test_tile_store_map_reads_the_k_major_core_matrix_layout():
    # operand of 128 rows x 64 bf16 features, K-major no-swizzle core matrices: row r, 8-feature
    # chunk c at (r // 8) * 1024 + c * 128 + (r % 8) * 16, feature f of the chunk at + 2 f
    def operand_offset(r, c, f):
        return (r // 8) * 1024 + c * 128 + (r % 8) * 16 + 2 * f

    rows_pad = 40 * 8  # a layer's rows, whole 8-row groups
    strides = [2, 128, 16, 1024, rows_pad * 128]  # bytes: feature, row, chunk, group, layer
    g0, layer = 5, 3  # the tile's first row group and its layer
    seen_smem, seen_global = set(), set()
    for k, (f, rr, c, g, z) in enumerate(box_order([8, 8, 8, 16, 1])):
        row = 8 * g + rr
        assert 2 * k == operand_offset(row, c, f)
        gaddr = f * strides[0] + rr * strides[1] + c * strides[2] + (g0 + g) * strides[3] + (layer + z) * strides[4]
        # the row-major [layer][row][64] bf16 element (layer, 8 g0 + row, 8 c + f)
        assert gaddr == ((layer * rows_pad + 8 * g0 + row) * 64 + 8 * c + f) * 2
        seen_smem.add(2 * k)
        seen_global.add(gaddr)
    assert len(seen_smem) == len(seen_global) == 128 * 64  # every element once


def test_output_gradient_map_lands_in_the_interleaved_mn_major_layout():
    # MN-major interleaved operand of a 32-record stage: 8 outputs (16 B) of record k in group g at
    # g * 512 + k * 16, i.e. 8-record core matrices 128 B apart (K) and groups 512 B apart (MN)
    def operand_offset(g, k, f):
        return g * 512 + (k // 8) * 128 + (k % 8) * 16 + 2 * f

    y = 64  # the stage's first record
    seen = set()
    for k, (f, rec, g) in enumerate(box_order([8, 32, 6])):
        assert 2 * k == operand_offset(g, rec, f)
        gaddr = f * 2 + (y + rec) * 96 + g * 16
        assert gaddr == ((y + rec) * 48 + 8 * g + f) * 2  # row-major [record][48] bf16
        seen.add(gaddr)
    assert len(seen) == 32 * 48


def test_swizzled_boxes_cover_the_operand_atoms():
    # the h / delta loads: boxes {64 features, 32 records, 5 layers} with the 128-byte swizzle,
    # one 128-byte row per record, 16-byte chunks XOR-permuted by the row's index in its 8-row group;
    # layer l's 4 KB then starts at l * 4096 (the A operand window of W_l, atom stride 4 KB)
    def swizzled(rec, chunk, layer):
        row = layer * 32 + rec
        return row * 128 + ((chunk ^ (row % 8)) * 16)

    offs = {swizzled(r, c, l) for l in range(5) for r in range(32) for c in range(8)}
    assert len(offs) == 5 * 32 * 8 and min(offs) == 0 and max(offs) == 5 * 4096 - 16
    for layer in range(5):
        block = {swizzled(r, c, layer) for r in range(32) for c in range(8)}
        assert min(block) == layer * 4096 and max(block) == layer * 4096 + 4096 - 16


def test_act_rows_padding_keeps_layers_apart():
    # layers are act_rows(n) = n rounded up to 8 rows apart, so a tile store's whole 8-row groups
    # never reach the next layer's rows
    def act_rows(n):
        return (n + 7) & ~7

    for n in [1, 7, 8, 33, 127, 128, 129, 65536, 65537]:
        rp = act_rows(n)
        assert rp % 8 == 0 and n <= rp < n + 8
        last_group_end = ((n - 1) // 8 + 1) * 8
        assert last_group_end <= rp
    assert np.array_equal([act_rows(n) for n in range(1, 17)], [8] * 8 + [16] * 8)
