"""The DIMACS reader (dmm_cnf_read) against a sequential restatement of its rules.

The C reader tokenizes the clause section in chunks on several threads (one chunk per MB);
the files here are large enough to be cut into several chunks, with comments, clauses that
span lines and chunk boundaries, and faults placed at random: the result, or the error
reported (the first in file order), must be the sequential reading's."""
import re
import zlib

import numpy as np
import pytest

import dmm_b200 as dmm

WS = b" \t\n\r\f\v"
INT_RE = re.compile(rb"^[+-]?[0-9]+$")
I64 = (-(1 << 63), (1 << 63) - 1)


TOKEN_RE = re.compile(rb"[^ \t\n\r\f\v]+")


def seq_read(data: bytes, path: str, max_lits: int = 25):
    """("ok", n, m, lits, off) or (status name, message): the rules of the reference's
    reader (dynex.cc:2306-2392) as the library states them, one token at a time."""
    it = TOKEN_RE.finditer(data)

    def token():
        return next(it, None)

    while True:
        t = token()
        if t is None:
            return ("DMM_ERR_PARSE", f"{path}: no `p cnf` header")
        if t.group() == b"p":
            break
    t = token()
    if t is None or t.group() != b"cnf":
        return ("DMM_ERR_PARSE", f"{path}: expected `p cnf n m`")
    n, m = int(token().group()), int(token().group())
    lits, off = [], [0]
    skip_to = -1  # a `c` token: tokens before the end of its line are skipped
    for ci in range(m):
        length = 0
        while True:
            t = token()
            if t is None:
                return ("DMM_ERR_PARSE", f"{path}: file ends after {ci} of {m} clauses")
            if t.start() < skip_to:
                continue
            tok = t.group()
            if tok == b"c":
                nl = data.find(b"\n", t.end())
                skip_to = len(data) if nl < 0 else nl
                continue
            if not INT_RE.match(tok):
                return ("DMM_ERR_PARSE", f"{path}: bad literal `{tok.decode()}` in clause {ci}")
            v = min(max(int(tok), I64[0]), I64[1])
            if v == 0:
                break
            if v > n or v < -n:
                return ("DMM_ERR_LITERAL", f"{path}: literal {v} out of range in clause {ci}")
            length += 1
            if length > max_lits:
                return ("DMM_ERR_CLAUSE_LEN", f"CLAUSE {ci} HAS MORE THAN {max_lits} LITERALS.")
            lits.append(v)
        off.append(len(lits))
    return ("ok", n, m, lits, off)


def make_file(rng, n, m, fault=None, fault_at=0.5, trailing=False):
    """A DIMACS text of m clauses over n variables with comment lines, `c` tokens inside
    lines, clauses broken over lines, tabs, CR-LF line ends and `+` signs; `fault` puts one
    defect at the clause fraction `fault_at`."""
    sizes = rng.integers(1, 8, size=m)
    total = int(sizes.sum())
    vals = rng.integers(1, n + 1, size=total) * rng.choice([-1, 1], size=total)
    plus = rng.random(total) < 0.05
    style = rng.random(m)
    strs = np.where(plus & (vals > 0), np.char.add("+", vals.astype(str)), vals.astype(str))
    starts = np.concatenate([[0], np.cumsum(sizes)])
    bad = int(fault_at * m)
    parts = ["c generated\n", "c key=101\n", f"p cnf {n} {m}\n"]
    for c in range(m):
        toks = list(strs[starts[c]:starts[c + 1]])
        if fault is not None and c == bad:
            j = len(toks) // 2
            if fault == "token":
                toks[j] = "1x2"
            elif fault == "range":
                toks[j] = str(n + 1 + c % 5)
            elif fault == "big":
                toks[j] = "-99999999999999999999999"
            elif fault == "long":
                toks = [str(1 + (c + i) % n) for i in range(26)]
        toks.append("0")
        r = style[c]
        if r < 0.02:
            parts.append("c a comment line 1 2 3\n")
        if r > 0.97:  # a clause over two lines, with a comment token in between
            h = len(toks) // 2
            parts.append(" ".join(toks[:h]) + " c inline 7 8\n" + "\t".join(toks[h:]) + "\n")
        elif r > 0.94:
            parts.append(" ".join(toks) + "\r\n")
        else:
            parts.append(" ".join(toks) + "\n")
    text = "".join(parts)
    if fault == "truncate":
        text = text[: int(len(text) * fault_at)]
        text = text[: text.rfind(" ")]  # a whole-token boundary
    if trailing:
        text += "1 2 zz 0\n" + str(10 * n) + " 0\n"
    return text.encode()


def check(tmp_path, data: bytes, name="f.cnf"):
    p = tmp_path / name
    p.write_bytes(data)
    want = seq_read(data, str(p))
    if want[0] == "ok":
        g = dmm.read_cnf(str(p))
        _, n, m, lits, off = want
        assert (g.n, g.m) == (n, m)
        assert np.array_equal(g.lits, np.array(lits, np.int32))
        assert np.array_equal(g.clause_off, np.array(off, np.int64))
        occ = np.bincount(np.abs(np.array(lits, np.int64)), minlength=n + 1)
        assert g.max_occurrence == (occ.max() if len(lits) else 0)
    else:
        with pytest.raises(dmm.DmmError) as e:
            dmm.read_cnf(str(p))
        assert e.value.name == want[0]
        assert want[1] in str(e.value)


@pytest.mark.parametrize("seed", [1, 2])
def test_reader_matches_sequential_rules_on_large_files(tmp_path, seed):
    rng = np.random.default_rng(seed)
    data = make_file(rng, 5000, 300_000)  # about 4.5 MB: several chunks
    assert len(data) > 3 << 20
    check(tmp_path, data)


@pytest.mark.parametrize("fault", ["token", "range", "big", "long", "truncate"])
@pytest.mark.parametrize("at", [0.0, 0.61])
def test_reader_reports_the_first_fault_in_file_order(tmp_path, fault, at):
    rng = np.random.default_rng(zlib.crc32(f"{fault}{at}".encode()))
    data = make_file(rng, 300, 150_000, fault=fault, fault_at=at)  # about 2 MB
    check(tmp_path, data)


def test_reader_ignores_what_follows_the_last_clause(tmp_path):
    rng = np.random.default_rng(7)
    check(tmp_path, make_file(rng, 300, 150_000, trailing=True))


def test_reader_small_and_empty_cases(tmp_path):
    for text in [b"p cnf 3 0\n", b"p cnf 3 0\n1 2 zz\n", b"p cnf 3 1\n0\n",
                 b"p cnf 3 2\n1 -2\n 3 0 -1 c x\n 0\n", b"p cnf 3 1\n-0\n", b"p cnf 3 1\n",
                 b"c only\n", b"p dnf 3 1\n1 0\n", b"p cnf 3 1\n1 2 3"]:
        check(tmp_path, text)


def test_writer_text_layout(tmp_path):
    """dmm_cnf_write: the planted comment line, the header, then one clause per line as
    `l1 l2 l3 0`, exactly; a large file reads back to the same formula."""
    f, planted = dmm.generate_planted(300, 1200, 0.08, 0.46, seed=3)
    p = str(tmp_path / "w.cnf")
    dmm.write_cnf(f, p, planted=planted)
    want = ("c [" + "".join(" %d" % (i + 1 if planted[i] > 0 else -(i + 1)) for i in range(300))
            + " ]\np cnf 300 1200\n"
            + "".join("".join("%d " % v for v in f.lits[f.clause_off[c]:f.clause_off[c + 1]]) + "0\n"
                      for c in range(1200)))
    assert open(p).read() == want
    big, _ = dmm.generate_planted(100_000, 420_000, 0.08, 0.46, seed=4)  # several MB: many blocks
    q = str(tmp_path / "big.cnf")
    dmm.write_cnf(big, q)
    g = dmm.read_cnf(q)
    assert np.array_equal(g.lits, big.lits) and np.array_equal(g.clause_off, big.clause_off)
