"""Oracle (test infrastructure only): restatement of the reference's dry run
of the local all-external loops, the records that drive them.

Only tests use this module; the product never imports it.

Restated (paths relative to ``tiger_ci/tiger_fortran``):
  all_external_3_4_loops_cho_2, first pass ... three_and_four_seg_mod_1.f90:414-436
      for a = num_internal+1 .. num_orbitals, c = num_internal+1 .. a
      (skipping ignorable_pair(c, a)), for every N-2 internal path in tree-search
      (lexical) order: build_ext_34seg_dryrun
  build_ext_34seg_dryrun ....................... three_and_four_seg_mod_1.f90:3142-3238
      skip_this_internal(head_weight, num_elec - 2) (locist_mod.f90:316-348: the
      path's internal_index_vector2 entry is negative), then the path's allowed
      virtuals (get_virtuals, num_allowed_virtuals) must hold both a and c; the
      record keeps icount = a (a - 1) / 2 + c, the head weight, the spin counts
      and the positions of a and c in the allowed-virtual list (from 1).
  ignorable_pair ............................... wp_tov_mod.f90:31-251: all false
      unless sphere-based integral truncation is on, which these decks do not use.

The record's CI addresses (internal_index_vector2 / 3 of the head, from 1) come
from the oracle's index vectors (sgga.build_space with per-path virtual counts).
"""
from __future__ import annotations

from . import sgga


def allext_records(deck: sgga.Deck, nm1_domains, nm2_domains):
    """Records (icount, head_weight, ab_address, aa_address, nsf_aa, nsf_ab, a_pos, c_pos), one per
    (external pair a >= c, N-2 path holding both); a domain [-1] marks a removed path. Addresses and spin
    counts are given only for a block that holds CSFs (0 otherwise)."""
    def nv(d):
        return 0 if list(d) == [-1] else len(d)

    sp = sgga.build_space(deck, [nv(d) for d in nm1_domains], [nv(d) for d in nm2_domains])
    nint, norb = deck.num_internal, deck.num_orbitals
    out = []
    for a in range(nint + 1, norb + 1):
        for c in range(nint + 1, a + 1):
            for p, h in enumerate(sp.paths[2]):
                dom = list(nm2_domains[p])
                # skip_this_internal: a removed path, or one without an ab index (killed)
                if dom == [-1] or h.get("off") is None:
                    continue
                virt = [nint + 1 + x for x in dom]  # get_virtuals: absolute orbital numbers, in order
                if a not in virt or c not in virt:
                    continue
                m = len(virt)
                has_ab = h["nsf"] > 0 and m >= 2
                has_aa = h.get("off_aa") is not None and h["nsf_aa"] > 0
                out.append((a * (a - 1) // 2 + c, h["lex"] - 1,
                            h["off"] + 1 if has_ab else 0, h["off_aa"] + 1 if has_aa else 0,
                            h["nsf_aa"] if has_aa else 0, h["nsf"] if has_ab else 0,
                            virt.index(a) + 1, virt.index(c) + 1))
    return out
