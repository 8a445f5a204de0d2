"""Oracle NM / MD:Z (nm_md_from_cigar, src/alignment/md.rs) pinned by the
reference's own cases: md.rs:213-282 and tests/md_format.rs:151-177."""
import pyoracle as O


def test_md_rs_known_answers():
    assert O.nm_md(b"ACGT", b"ACGT", 0, 0, [(4, "M")]) == (0, "4")                    # :214
    assert O.nm_md(b"ACGT", b"AGGT", 0, 0, [(4, "M")]) == (1, "1G2")                  # :220
    assert O.nm_md(b"TTGA", b"ACGT", 0, 0, [(4, "M")]) == (3, "0A0C1T0")              # :226
    assert O.nm_md(b"ACGTACGT", b"ACGTTTACGT", 0, 0,
                   [(3, "M"), (2, "D"), (5, "M")]) == (2, "3^TT5")                    # :232
    assert O.nm_md(b"ACGAAGTA", b"ACGGTA", 0, 0,
                   [(3, "M"), (2, "I"), (3, "M")]) == (2, "6")                        # :239
    assert O.nm_md(b"NNACGN", b"XXXXACG", 0, 4,
                   [(2, "S"), (3, "M"), (1, "S")]) == (0, "3")                        # :250
    ref = bytearray(b"T" * 104)
    ref[0:2] = b"AC"
    ref[102:104] = b"GA"
    assert O.nm_md(b"ACGA", bytes(ref), 0, 0,
                   [(2, "M"), (100, "N"), (2, "M")]) == (0, "4")                      # :262


def test_md_builder_cases():
    # md.rs:276-281: columns(ACGT, ACCT) then insertion(2)
    assert O.md_builder("CCCCI", b"ACGT", b"ACCT", [0, 0, 0, 0, 2]) == (3, "2C1")
    # md_format.rs:151-160: mismatch(0xff), deletion(r 0 ^ 0xc3 0xa9), deletion([]), matched()
    nm, md = O.md_builder("XDDM", b"", bytes([0xFF, ord("r"), 0, ord("^"), 0xC3, 0xA9]),
                          [0, 5, 0, 0])
    assert (nm, md) == (6, "0N0^RNNNN1")
    # md_format.rs:166-167: ambiguity and case rules
    assert O.md_builder("CCCCC", b"aNr=A", b"ANRNC") == (3, "4C0")


def test_past_the_ends_and_deletion_overhang():
    # positions past either end read as N; deleted bases past the reference end
    # still count toward NM (md.rs:172-194)
    assert O.nm_md(b"AC", b"AC", 0, 0, [(3, "M")]) == (1, "3")   # N vs N: run + 1, NM + 1
    nm, md = O.nm_md(b"ACGT", b"ACG", 0, 0, [(3, "M"), (4, "D")])
    assert (nm, md) == (4, "3")
