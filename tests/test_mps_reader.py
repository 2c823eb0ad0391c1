"""MPS reader (pdhg_read_mps): the reference's read_mps_string, field by field.

Every case is read by the engine library and, where oracle/_ref is built, by
the reference's own reader (src/io/mps_reader.cpp, compiled unmodified): the
arrays must be bit-identical, and the names, integrality, warnings (line,
section, text) and error messages identical. The cases cover each dialect
rule the reference handles (sections, row types, RANGES by row type, every
bound type, infinite spellings, integer markers, OBJSENSE forms, comments and
CRLF, the fixed-column retry, unsupported sections, malformed cards), seeded
random models written with all of them, and models whose COLUMNS section is
large enough to be parsed by threads in chunks.
"""
import numpy as np
import pytest

ARRAYS = ("row_ptr", "col_idx", "val", "c", "col_lo", "col_hi", "row_lo", "row_hi")


def ours(pkg, text, **kw):
    try:
        return pkg.mps.read_mps(text, **kw)
    except pkg.mps.MpsError as e:
        return str(e)


def same_as_reference(pkg, orc, text, origin=None, keep_lower_at_zero=False, keep_free_rows=True,
                      threads=0):
    a = ours(pkg, text, origin=origin,
             negative_upper_bound="keep_lower_at_zero" if keep_lower_at_zero else "minus_infinity",
             keep_free_rows=keep_free_rows, threads=threads)
    if not orc.ref_available():
        return a
    b = orc.reference_read_mps(text, origin if origin is not None else "<string>",
                               keep_lower_at_zero, keep_free_rows)
    if "error" in b:
        assert isinstance(a, str), (a, b["error"])
        assert a == b["error"]
        return a
    assert not isinstance(a, str), (a, b)
    p = a.problem
    assert (p.m, p.n, p.maximize) == (b["m"], b["n"], b["maximize"])
    assert p.obj_const == b["obj_const"] or (np.isnan(p.obj_const) and np.isnan(b["obj_const"]))
    for f in ARRAYS:
        x, y = getattr(p, f), b[f]
        assert x.dtype == y.dtype and x.shape == y.shape, f
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f  # bit for bit
    assert np.array_equal(a.is_integer, b["is_integer"])
    assert (a.name, a.objective_name) == (b["name"], b["objective_name"])
    assert a.row_names == b["row_names"] and a.col_names == b["col_names"]
    assert a.warnings == b["warnings"]
    assert a.fixed_format == any(w[1] == "FORMAT" for w in b["warnings"])
    return a


BASIC = """NAME          SMALL
ROWS
 N  COST
 L  CAP
 G  NEED
 E  BAL
COLUMNS
    X1        COST         1.0   CAP          1.0
    X1        NEED         1.0
    X2        COST         2.0   CAP          1.0
    X2        BAL         -1.0
    X3        COST        -1.0   BAL          1.0
RHS
    RHS       COST        -3.5
    RHS       CAP          4.0   NEED         1.0
    RHS       BAL          7.0
RANGES
    RNG       CAP          2.5   BAL         -3.0
BOUNDS
 UP BND       X1           4.0
 MI BND       X2
 UP BND       X3          -2.0
ENDATA
"""


def test_basic_model_known_answer(pkg, orc):
    a = same_as_reference(pkg, orc, BASIC)
    p = a.problem
    assert (p.m, p.n, p.nnz, a.name, a.objective_name) == (3, 3, 5, "SMALL", "COST")
    assert a.row_names == ["CAP", "NEED", "BAL"] and a.col_names == ["X1", "X2", "X3"]
    assert list(p.c) == [1.0, 2.0, -1.0] and p.obj_const == 3.5  # RHS on the objective: -d
    # L row with range 2.5: [4 - 2.5, 4]; G row: [1, inf); E row with range -3: [7 - 3, 7]
    assert list(p.row_lo) == [1.5, 1.0, 4.0] and list(p.row_hi) == [4.0, np.inf, 7.0]
    # UP 4; MI; UP -2 on a default-zero lower bound frees it below (with a warning)
    assert list(p.col_lo) == [0.0, -np.inf, -np.inf] and list(p.col_hi) == [4.0, np.inf, -2.0]
    assert a.warnings[0][0] == 22 and a.warnings[0][1] == "BOUNDS"
    # the literal reading keeps the crossed pair, which fails validation
    e = same_as_reference(pkg, orc, BASIC, keep_lower_at_zero=True)
    assert isinstance(e, str) and "crossed bounds on column X3" in e


def card(*fields):
    return "    " + "   ".join(fields)


def model(rows, columns, rhs=(), ranges=(), bounds=(), head="NAME T\n", tail="ENDATA\n"):
    out = [head.rstrip("\n")] if head else []
    out.append("ROWS")
    out += [f" {t}  {n}" for t, n in rows]
    out.append("COLUMNS")
    out += [card(*c) for c in columns]
    if rhs:
        out.append("RHS")
        out += [card(*r) for r in rhs]
    if ranges:
        out.append("RANGES")
        out += [card(*r) for r in ranges]
    if bounds:
        out.append("BOUNDS")
        out += [" " + "  ".join(b) for b in bounds]
    return "\n".join(out) + "\n" + tail


ROWS3 = [("N", "obj"), ("L", "r1"), ("G", "r2"), ("E", "r3")]


def test_each_dialect_rule_matches_the_reference(pkg, orc):
    cases = {
        # a second N row is a free row, not a second objective; dropping it
        "free_row": model(ROWS3 + [("N", "spare")],
                          [("x", "obj", "1", "spare", "5", "r1", "1"), ("y", "r2", "1", "r3", "2")],
                          rhs=[("RHS", "spare", "3"), ("r1", "4")], ranges=[("R", "spare", "1")]),
        # duplicates sum in file order, zero sums vanish, rows order by column
        "duplicates": model(ROWS3, [("b", "r1", "1.5"), ("a", "r1", "2", "r2", "1e-15"),
                                    ("b", "r1", "-1.5", "r3", "0.1"), ("a", "r1", "0.25"),
                                    ("b", "r3", "0.2"), ("a", "r3", "0.7")]),
        # ranges: |R| on L and G rows, the signed R on E rows
        "ranges": model(ROWS3 + [("E", "r4")],
                        [("x", "r1", "1", "r2", "1"), ("y", "r3", "1", "r4", "1")],
                        rhs=[("B", "r1", "10"), ("B", "r2", "-2"), ("B", "r3", "5"), ("B", "r4", "5")],
                        ranges=[("R", "r1", "-4"), ("R", "r2", "-3"), ("R", "r3", "2"), ("R", "r4", "-2")]),
        # every bound type, in both cases of spelling
        "bounds": model(ROWS3, [(f"c{k}", "r1", "1") for k in range(10)],
                        bounds=[("UP", "B", "c0", "3"), ("lo", "B", "c1", "-2"), ("FX", "B", "c2", "1.5"),
                                ("FR", "B", "c3"), ("MI", "B", "c4"), ("PL", "B", "c5"),
                                ("BV", "B", "c6"), ("LI", "B", "c7", "2"), ("UI", "B", "c8", "9"),
                                ("UP", "c9", "4")]),
        # infinite spellings: INF, -Infinity, 1e30 and beyond
        "infinities": model(ROWS3, [(f"c{k}", "r1", "1") for k in range(6)],
                            bounds=[("UP", "B", "c0", "INF"), ("LO", "B", "c1", "-Infinity"),
                                    ("UP", "B", "c2", "1e30"), ("LO", "B", "c3", "-1e31"),
                                    ("UP", "B", "c4", "+inf"), ("LO", "B", "c5", "-9.99e29")]),
        # integer markers, quoted or not, and a bound on a column without coefficients
        "markers": model(ROWS3, [("x", "r1", "1"), ("M1", "'MARKER'", "'INTORG'"), ("i1", "r1", "1"),
                                 ("i2", "r2", "1"), ("M2", "'MARKER'", "'INTEND'"), ("y", "r3", "1"),
                                 ("M3", "marker", "intorg"), ("i3", "r3", "2"), ("M4", "MARKER", "INTEND")],
                         bounds=[("UP", "B", "i1", "5"), ("UP", "B", "ghost", "2")]),
        # OBJSENSE on its own card, then inline
        "objsense_card": "NAME X\nOBJSENSE\n    MAX\n" + model(ROWS3, [("x", "obj", "1", "r1", "1")], head=""),
        "objsense_inline": "OBJSENSE MAXIMIZE\n" + model(ROWS3, [("x", "obj", "1", "r1", "1")], head=""),
        # comments, CRLF, tabs, blank lines, lines after ENDATA
        "crlf": model(ROWS3, [("x", "obj", "2", "r1", "1")]).replace("\n", "\r\n").replace(
            "COLUMNS", "* a comment\r\n\r\nCOLUMNS") + "garbage after the end\n",
        "tabs": model(ROWS3, [("x", "obj", "2", "r1", "1")]).replace("    ", "\t"),
        # unsupported sections are reported and skipped
        "qsection": model(ROWS3, [("x", "obj", "2", "r1", "1")], tail="QSECTION obj\n    x x 1\nENDATA\n"),
        # RHS without a set name, an odd card with a set name, pairs on one card
        "rhs_forms": model(ROWS3, [("x", "r1", "1", "r2", "1"), ("y", "r3", "1")],
                           rhs=[("r1", "1", "r2", "2"), ("SET", "r3", "3")]),
        # number spellings strtod takes
        "numbers": model(ROWS3, [("x", "r1", "+2", "r2", "4."), ("y", "r1", ".5", "r3", "1E+2"),
                                 ("z", "r2", "-3e-2", "r3", "0x1p-2")]),
        # no ENDATA at all
        "no_endata": model(ROWS3, [("x", "obj", "1", "r1", "1")], tail=""),
        "upper_bound_default_then_lo": model(ROWS3, [("x", "r1", "1")],
                                             bounds=[("UP", "B", "x", "-1"), ("LO", "B", "x", "-5")]),
    }
    for name, text in cases.items():
        r = same_as_reference(pkg, orc, text)
        assert not isinstance(r, str), (name, r)
    # free rows dropped on request
    r = same_as_reference(pkg, orc, cases["free_row"], keep_free_rows=False)
    assert not isinstance(r, str) and r.problem.m == 3
    # known answers that hold without the reference
    d = ours(pkg, cases["duplicates"]).problem
    assert list(d.row_ptr) == [0, 1, 1, 3] and list(d.col_idx) == [1, 0, 1]  # (b, r1) cancels; 1e-15 drops
    assert list(d.val) == [2.25, 0.1 + 0.2, 0.7]
    rg = ours(pkg, cases["ranges"]).problem
    assert list(rg.row_lo) == [6, -2, 5, 3] and list(rg.row_hi) == [10, 1, 7, 5]
    mk = ours(pkg, cases["markers"])
    assert list(mk.is_integer) == [False, True, True, False, True, False]
    assert mk.col_names[-1] == "ghost"
    assert ours(pkg, cases["objsense_card"]).problem.maximize
    assert ours(pkg, cases["numbers"]).problem.val[-1] == 0.25


def fixed_card(*fields):
    """A data card in the fixed layout: fields at card columns 2, 5, 15, 25, 40, 50."""
    line = [" "] * 61
    for start, f in zip((1, 4, 14, 24, 39, 49), fields):
        line[start:start + len(f)] = list(f)
    return "".join(line).rstrip()


def test_fixed_column_names_with_spaces_take_the_retry(pkg, orc):
    # names with embedded blanks only parse under the fixed card layout
    text = "\n".join([
        "NAME          FIXED", "ROWS", fixed_card("N", "COST"), fixed_card("L", "LIM 1"),
        fixed_card("L", "LIM 2"), "COLUMNS",
        fixed_card("", "X ONE", "COST", "1.0", "LIM 1", "1.0"),
        fixed_card("", "X ONE", "LIM 2", "2.0"),
        fixed_card("", "X TWO", "COST", "-1.0", "LIM 2", "1.0"),
        "RHS", fixed_card("", "RHS", "LIM 1", "4.0", "LIM 2", "6.0"),
        "BOUNDS", fixed_card("UP", "BND", "X TWO", "3.5"), "ENDATA"]) + "\n"
    a = same_as_reference(pkg, orc, text)
    assert not isinstance(a, str), a
    assert a.fixed_format and a.warnings[0][:2] == (0, "FORMAT")
    assert a.row_names == ["LIM 1", "LIM 2"] and a.col_names == ["X ONE", "X TWO"]
    assert list(a.problem.row_hi) == [4.0, 6.0] and a.problem.col_hi[1] == 3.5
    # the same model with one-word names is read free-form, without the note
    plain = text.replace("LIM 1", "LIM1 ").replace("LIM 2", "LIM2 ").replace(
        "X ONE", "XONE ").replace("X TWO", "XTWO ")
    b = same_as_reference(pkg, orc, plain)
    assert not b.fixed_format and not b.warnings


def test_malformed_models_fail_with_the_reference_message(pkg, orc):
    bad = [
        "",
        "ROWS\n L r\nCOLUMNS\n x r 1\n",                              # no N row
        " x r 1\n",                                                    # data before any section
        "ROWS\n N c\n Q r\n",                                          # unknown row type
        "ROWS\n N c\n L r\n L r\n",                                    # duplicate row
        "ROWS\n N c\n L\n",                                            # short ROWS card
        "ROWS\n N c\n L r\nCOLUMNS\n x r\n",                           # short COLUMNS card
        "ROWS\n N c\n L r\nCOLUMNS\n x r one\n",                       # not a number
        "ROWS\n N c\n L r\nCOLUMNS\n x q 1\n",                         # unknown row
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nRHS\n B q 1\n",            # unknown row in RHS
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nRANGES\n B q 1\n",         # unknown row in RANGES
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nBOUNDS\n UP B x\n",        # bound without value
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nBOUNDS\n XX B x 1\n",      # unknown bound type
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nBOUNDS\n SC B x 1\n",      # semi-continuous
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nBOUNDS\n UP\n",            # short BOUNDS card
        "OBJSENSE\n    UP\nROWS\n N c\n",                             # unknown sense
        "ROWS\n N c\n L r\nCOLUMNS\n x r inf\n",                       # infinite coefficient
        "ROWS\n N c\n L r\nCOLUMNS\n x r nan\n",                       # NaN coefficient
        "ROWS\n N c\n L r\nCOLUMNS\n x c nan r 1\n",                   # NaN objective
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nRHS\n B r nan\n",          # NaN row bound
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nRHS\n B c inf\n",          # infinite constant
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nBOUNDS\n LO B x 5\n UP B x 4\n",  # crossed
        "ROWS\n N c\n L r\nCOLUMNS\n M 'MARKER' 'INTORG'\n x r 1\nBOUNDS\n UP B x 2.5\n",  # fractional
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nRHS\n B r\n",              # short RHS card
        "ROWS\n N c\n L r\nCOLUMNS\n x r 1\nRANGES\n R\n",             # short RANGES card
    ]
    for text in bad:
        r = same_as_reference(pkg, orc, text)
        assert isinstance(r, str), text
    assert ours(pkg, bad[1]) == "<string>: no objective row (no N row in the ROWS section)"
    assert ours(pkg, bad[8]) == "<string>:5: unknown row 'q' in COLUMNS"
    assert ours(pkg, bad[16]) == "from_triplets: non-finite coefficient"
    assert ours(pkg, bad[4]) == "duplicate row name 'r'"
    r = same_as_reference(pkg, orc, bad[8], origin="model.mps")
    assert r == "model.mps:5: unknown row 'q' in COLUMNS"


def test_file_entry_point(pkg, orc, tmp_path):
    f = tmp_path / "small.mps"
    f.write_text(BASIC)
    a = pkg.mps.read_mps_file(str(f))
    b = pkg.mps.read_mps(BASIC)
    for k in ARRAYS:
        assert np.array_equal(getattr(a.problem, k), getattr(b.problem, k))
    with pytest.raises(pkg.mps.MpsError, match="cannot open"):
        pkg.mps.read_mps_file(str(tmp_path / "missing.mps"))
    # a file's errors name the file, like read_mps(path)
    g = tmp_path / "bad.mps"
    g.write_text("ROWS\n N c\n L r\nCOLUMNS\n x q 1\n")
    with pytest.raises(pkg.mps.MpsError, match=f"{g}:5: unknown row 'q' in COLUMNS"):
        pkg.mps.read_mps_file(str(g))


# ---- seeded models written with every rule -------------------------------------------------

NUM_FORMS = ("{:.17g}", "{:.6f}", "{:+.3e}", "{:.4E}")


def fmt(rng, v):
    if v == int(v) and abs(v) < 1e6 and rng.random() < 0.3:
        return str(int(v)) + ("." if rng.random() < 0.3 else "")
    return NUM_FORMS[rng.integers(len(NUM_FORMS))].format(v)


def write_random_mps(seed, m=30, n=60, big=False, bounds_p=0.4, ghosts=0):
    """A random model in free MPS with the dialect's quirks; when big, many
    columns (a COLUMNS section of several MB) for the chunked parse."""
    rng = np.random.default_rng(seed)
    nl = "\r\n" if rng.random() < 0.2 else "\n"
    sep = "\t" if rng.random() < 0.2 else "  "
    L = []
    if rng.random() < 0.7:
        L.append(f"NAME {'M' + str(seed)}")
    if rng.random() < 0.3:
        L += ["OBJSENSE", "    MAX"] if rng.random() < 0.5 else ["OBJSENSE MIN"]
    L.append("ROWS")
    L.append(" N obj")
    types = rng.choice(["L", "G", "E", "l", "e"], size=m)
    for i in range(m):
        L.append(f" {types[i]} r{i}")
    if rng.random() < 0.3:
        L.append(" N free0")
    L.append("COLUMNS")
    in_int = False
    for j in range(n):
        if rng.random() < 0.05:
            in_int = not in_int
            q = "'" if rng.random() < 0.7 else ""
            L.append(f"    MK{j}{sep}{q}MARKER{q}{sep}{q}{'INTORG' if in_int else 'INTEND'}{q}")
        k = int(rng.integers(1, 5))
        rows = rng.choice(m, size=k, replace=True)  # repeats: duplicates that sum
        pairs = [(f"r{r}", fmt(rng, float(np.round(rng.standard_normal(), 3)))) for r in rows]
        if rng.random() < 0.6:
            pairs.append(("obj", fmt(rng, float(np.round(rng.standard_normal(), 2)))))
        if rng.random() < 0.02:
            pairs.append(("free0" if " N free0" in L else "obj", "1"))
        rng.shuffle(pairs)
        q = 0
        while q < len(pairs):
            take = 2 if (rng.random() < 0.5 and q + 1 < len(pairs)) else 1
            body = sep.join(f"{a}{sep}{b}" for a, b in pairs[q:q + take])
            L.append(f"    x{j}{sep}{body}")
            q += take
        if rng.random() < 0.01:
            L.append("* comment inside COLUMNS")
        if rng.random() < 0.01:
            L.append("")
    L.append("RHS")
    for i in range(m):
        if rng.random() < 0.7:
            L.append(f"    {'RHS' + sep if rng.random() < 0.5 else ''}r{i}{sep}{fmt(rng, float(rng.integers(-5, 6)))}")
    if rng.random() < 0.5:
        L.append(f"    RHS{sep}obj{sep}{fmt(rng, 2.5)}")
    if rng.random() < 0.7:
        L.append("RANGES")
        for i in range(m):
            if rng.random() < 0.3:
                L.append(f"    RNG{sep}r{i}{sep}{fmt(rng, float(rng.integers(-4, 5)))}")
    L.append("BOUNDS")
    kinds = ["UP", "LO", "FX", "FR", "MI", "PL", "BV", "LI", "UI", "up"]
    for j in range(n):
        if ghosts and rng.random() < ghosts / n:  # columns COLUMNS never named, some twice
            g = int(rng.integers(ghosts))
            L.append(f" UP BND ghost{g} {fmt(rng, float(rng.integers(0, 9)))}")
        if rng.random() < bounds_p:
            t = kinds[int(rng.integers(len(kinds)))]
            if t in ("FR", "MI", "PL", "BV"):
                L.append(f" {t} BND x{j}")
            else:
                v = float(rng.integers(-3, 10))
                if t == "UI":
                    v = abs(v)  # UI does not free the lower end: a negative one would cross
                if t in ("UP", "up") and rng.random() < 0.1:
                    vs = ["inf", "1e30", "-1e30", "+INF", "Infinity"][int(rng.integers(5))]
                else:
                    vs = fmt(rng, v)
                L.append(f" {t} BND x{j} {vs}")
    if rng.random() < 0.3:
        L.append(" UP BND ghost 4")
    if rng.random() < 0.8:
        L.append("ENDATA")
    return nl.join(L) + nl


@pytest.mark.parametrize("seed", range(40))
def test_random_models_match_the_reference(pkg, orc, seed):
    text = write_random_mps(seed)
    same_as_reference(pkg, orc, text)
    same_as_reference(pkg, orc, text, keep_lower_at_zero=True, keep_free_rows=False)


@pytest.mark.parametrize("seed", [100, 101, 102])
def test_large_columns_sections_parse_in_chunks(pkg, orc, seed):
    # a COLUMNS section of several MB goes to the threads in chunks; the model
    # must not depend on the thread count and must match the reference
    text = write_random_mps(seed, m=400, n=60_000)
    assert len(text) > 3_000_000
    a = same_as_reference(pkg, orc, text, threads=8)
    assert not isinstance(a, str), a
    assert a.problem.nnz > 100_000 and a.is_integer.any()
    one = ours(pkg, text, threads=1)
    for f in ARRAYS:
        assert np.array_equal(getattr(one.problem, f), getattr(a.problem, f))
    assert one.col_names == a.col_names and np.array_equal(one.is_integer, a.is_integer)
    assert one.warnings == a.warnings


def test_chunked_parse_reports_the_first_error_with_its_line(pkg, orc):
    text = write_random_mps(7, m=50, n=50_000)
    head, _, rest = text.partition("RHS")
    lines = head.split("\n")
    # two errors deep in COLUMNS: the earlier one is the one reported
    k1, k2 = len(lines) * 2 // 3, len(lines) * 5 // 6
    lines[k1] = "    x1 nosuchrow 1"
    lines[k2] = "    x2 r1 notanumber"
    text = "\n".join(lines) + "RHS" + rest
    r = same_as_reference(pkg, orc, text, threads=8)
    assert r == ours(pkg, text, threads=1)
    assert isinstance(r, str) and f":{k1 + 1}: unknown row 'nosuchrow' in COLUMNS" in r


@pytest.mark.parametrize("maker", ["random_equality", "badly_scaled", "mixed_bounds", "transportation"])
def test_written_models_read_back(pkg, orc, maker):
    # write_mps then read_mps returns the model (ranges up to hi - lo's rounding)
    from conftest import golden_problem, load_golden
    p = {"random_equality": lambda: pkg.lpgen.random_equality_lp(40, 90, 4, seed=3, maximize=True),
         "badly_scaled": lambda: pkg.lpgen.badly_scaled_lp(50, 120, 5, seed=4),
         "mixed_bounds": lambda: golden_problem(pkg, load_golden("mixed_bounds_50x90")),
         "transportation": lambda: pkg.lpgen.transportation_lp(20, 30, seed=5)}[maker]()
    p.obj_const = 1.25
    text = pkg.mps.write_mps(p)
    a = same_as_reference(pkg, orc, text)
    q = a.problem
    for f in ("row_ptr", "col_idx", "val", "c", "col_lo", "col_hi", "row_lo"):
        assert np.array_equal(getattr(q, f), getattr(p, f)), f
    ranged = np.isfinite(p.row_lo) & np.isfinite(p.row_hi) & (p.row_lo != p.row_hi)
    assert np.array_equal(q.row_hi[~ranged], p.row_hi[~ranged])
    assert np.allclose(q.row_hi[ranged], p.row_hi[ranged], rtol=1e-15, atol=0)
    assert (q.obj_const, q.maximize) == (p.obj_const, p.maximize)


def test_cpp_reader_adapter_matches_the_reference(tmp_path):
    """sov::MpsModelB200 (include/pdhg_b200_sov.hpp) against the reference's
    sov::read_mps, as C++ callers see them: oracle/_ref/mps_check reads every
    file with both, under both negative-upper-bound rules, and compares the
    sov::ReadResult field by field (or the sov::Error text)."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "oracle", "_ref", "mps_check")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/mps_check not built (needs the reference sources)")
    texts = {"basic": BASIC,
             "fixed": "\n".join([
                 "NAME          FIXED", "ROWS", fixed_card("N", "COST"), fixed_card("L", "LIM 1"),
                 "COLUMNS", fixed_card("", "X ONE", "COST", "1.0", "LIM 1", "1.0"),
                 "RHS", fixed_card("", "RHS", "LIM 1", "4.0"), "ENDATA"]) + "\n",
             "markers": model(ROWS3, [("x", "r1", "1"), ("M1", "'MARKER'", "'INTORG'"),
                                      ("i1", "r1", "1"), ("M2", "'MARKER'", "'INTEND'")],
                              bounds=[("UP", "B", "i1", "5"), ("UP", "B", "ghost", "2")]),
             "bad_row": "ROWS\n N c\n L r\nCOLUMNS\n x q 1\n",
             "no_objective": "ROWS\n L r\nCOLUMNS\n x r 1\n"}
    for seed in range(10):
        texts[f"random{seed}"] = write_random_mps(seed)
    files = []
    for name, text in texts.items():
        f = tmp_path / f"{name}.mps"
        f.write_text(text)
        files.append(str(f))
    r = subprocess.run([exe] + files, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ALL OK" in r.stdout, r.stdout[-3000:] + r.stderr[-2000:]


def test_bench_mps_reader_line():
    """bench.py --mps-reader prints one JSON line: the reader's throughput on a
    written transportation model, one thread and all, and the reference's
    reader on a sample when oracle/_ref is built."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--mps-reader",
                        "--supplies", "30", "--demands", "60", "--mps-ref-supplies", "10"],
                       capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-3000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["metric"] == "mps_read_throughput" and line["unit"] == "MB/s"
    assert line["value"] > 0 and line["single_thread_MBps"] > 0
    assert line["config"]["nonzeros"] == 2 * 30 * 60 and line["config"]["columns"] == 30 * 60
    ref = line["reference"]
    assert "unavailable" in ref or (ref["value"] > 0 and ref["kind"] == "reference")


@pytest.mark.parametrize("seed", [200, 201])
def test_large_bounds_sections_parse_in_chunks(pkg, orc, seed):
    # a BOUNDS card on every column (a section of more than 1 MB) goes to the
    # threads in chunks and is applied in file order: bounds on columns COLUMNS
    # never named (the first makes the column and warns), negative UP bounds
    # under both rules, every bound type
    text = write_random_mps(seed, m=300, n=60_000, bounds_p=1.0, ghosts=40)
    assert len(text.partition("BOUNDS")[2]) > 1_100_000
    for lit in (False, True):
        a = same_as_reference(pkg, orc, text, keep_lower_at_zero=lit, threads=8)
        one = ours(pkg, text, threads=1,
                   negative_upper_bound="keep_lower_at_zero" if lit else "minus_infinity")
        if isinstance(a, str):
            assert one == a
            continue
        assert any(w[2].startswith("bound on column 'ghost") for w in a.warnings)
        for f in ARRAYS:
            assert np.array_equal(getattr(one.problem, f), getattr(a.problem, f))
        assert one.col_names == a.col_names and one.warnings == a.warnings
        assert np.array_equal(one.is_integer, a.is_integer)


def test_chunked_bounds_report_the_first_error_with_its_line(pkg, orc):
    text = write_random_mps(9, m=100, n=60_000, bounds_p=1.0)
    head, _, rest = text.partition("BOUNDS")
    lines = rest.split("\n")
    k1, k2 = len(lines) * 2 // 3, len(lines) * 5 // 6
    lines[k1] = " UP BND x5 notanumber"
    lines[k2] = " XX BND x6 1"
    text = head + "BOUNDS" + "\n".join(lines)
    r = same_as_reference(pkg, orc, text, threads=8)
    assert r == ours(pkg, text, threads=1)
    assert isinstance(r, str) and "expected a number, got 'notanumber'" in r


FUZZ_ALPHABET = list(" \t\r\n*'+-.eE0123456789ABCDEFGHIJKLMNOPQRSTUVWXYZabcxyz") + [
    "INF", "MARKER", "'INTORG'", "RHS", "ROWS", "BOUNDS", "COLUMNS", "RANGES", "N", "UP", "FR"]


def mutate(rng, s):
    """One to four random edits: a character deleted, inserted or replaced
    (from MPS's own vocabulary), a line duplicated or two lines swapped."""
    for _ in range(rng.randint(1, 4)):
        if not s:
            s = "x"
        i = rng.randrange(len(s))
        op = rng.random()
        if op < 0.3:
            s = s[:i] + s[i + 1:]
        elif op < 0.6:
            s = s[:i] + rng.choice(FUZZ_ALPHABET) + s[i:]
        elif op < 0.8:
            s = s[:i] + rng.choice(FUZZ_ALPHABET) + s[i + 1:]
        else:
            lines = s.split("\n")
            a, b = rng.randrange(len(lines)), rng.randrange(len(lines))
            if rng.random() < 0.5:
                lines.insert(b, lines[a])
            else:
                lines[a], lines[b] = lines[b], lines[a]
            s = "\n".join(lines)
    return s


def test_mutated_models_read_like_the_reference(pkg, orc):
    # seeded byte-level mutations of valid free and fixed-layout models: the
    # two readers must agree on every one (the same error text or the same
    # model, warnings included)
    import random
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    fixed = "\n".join([
        "NAME          FIXED", "ROWS", fixed_card("N", "COST"), fixed_card("L", "LIM 1"),
        fixed_card("G", "LIM 2"), "COLUMNS", fixed_card("", "X ONE", "COST", "1.0", "LIM 1", "1.0"),
        fixed_card("", "X ONE", "LIM 2", "2.0"), fixed_card("", "X TWO", "COST", "-1.0", "LIM 2", "1.0"),
        "RHS", fixed_card("", "RHS", "LIM 1", "4.0", "LIM 2", "1.0"),
        "RANGES", fixed_card("", "RNG", "LIM 1", "2.5"),
        "BOUNDS", fixed_card("UP", "BND", "X TWO", "3.5"), fixed_card("MI", "BND", "X ONE"),
        "ENDATA"]) + "\n"
    bases = [BASIC, fixed, fixed.replace("\n", "\r\n")] + [write_random_mps(s, m=6, n=10) for s in range(8)]
    rng = random.Random(2024)
    models = 0
    for _ in range(600):
        text = mutate(rng, rng.choice(bases))
        for lit in (False, True):
            r = same_as_reference(pkg, orc, text, keep_lower_at_zero=lit)
            models += not isinstance(r, str)
    assert models > 100  # the mutations leave many models readable
