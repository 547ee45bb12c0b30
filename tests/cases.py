"""Shared small MRSDCI test spaces (orbitals, internal split, electrons, spin,
references, frozen) covering singlet/doublet/triplet/quintet, several
references, open-shell references and frozen orbitals."""
SMALL_CASES = [
    dict(no=6, ni=2, na=1, ne=4, sm=1, refs=["220"]),
    dict(no=6, ni=3, na=0, ne=6, sm=1, refs=["222"]),
    dict(no=7, ni=2, na=2, ne=6, sm=1, refs=["2220", "2202"]),
    dict(no=7, ni=2, na=2, ne=6, sm=3, refs=["2211"]),
    dict(no=7, ni=2, na=2, ne=5, sm=2, refs=["2210", "2201"]),
    dict(no=8, ni=1, na=4, ne=6, sm=1, refs=["22110", "21111", "22200"]),
    dict(no=8, ni=2, na=3, ne=6, sm=5, refs=["21111"]),
    dict(no=8, ni=3, na=1, ne=8, sm=1, refs=["2222"], nf=1),
    dict(no=9, ni=2, na=3, ne=8, sm=1, refs=["22220", "22202", "22022", "22121"]),
    dict(no=8, ni=2, na=2, ne=6, sm=3, refs=["2211", "2121"], nf=1),
]


def case_id(c):
    return f"no{c['no']}-ni{c['ni']}-na{c['na']}-e{c['ne']}-m{c['sm']}-r{len(c['refs'])}" + (f"-f{c['nf']}" if c.get("nf") else "")


def product_deck(c):
    import tigerci_b200 as T

    return T.Deck(c["no"], c["ni"], c["na"], c["ne"], c["sm"], c["refs"], num_frozen=c.get("nf", 0))


def oracle_deck(c):
    from oracle import sgga

    return sgga.Deck(c["no"], c["ni"], c["na"], c["ne"], c["sm"], c["refs"], c.get("nf", 0))
