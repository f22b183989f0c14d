"""Text cases for the .tns loader tests (shared by the CPU oracle pin and the
GPU parser test)."""
import numpy as np

CASES = {
    "plain": b"3 6\n1 2 3 1.5\n3 2 1 2.25\n5 5 1 1e-3\n",
    "no_trailing_newline": b"3 6\n1 2 3 1.5\n3 2 1 2.25\n5 5 1 1e-3",
    "crlf_tabs_blank_lines": b"\r\n3\t6\r\n\r\n1  2\t3   1.5\r\n\t3 2 1 2.25\r\n5 5 1 -7\r\n\r\n",
    "partial_record": b"3 6\n1 2 3 1.5\n3 2 1 2.25\n5 5\n",
    "one_line": b"3 6 1 2 3 1.5 4 4 4 2.5 ",
    "value_forms": (b"2 9\n1 1 +1.5\n1 2 .5\n1 3 5.\n1 4 5.e3\n1 5 -0.0\n1 6 1E-5\n1 7 0.000123\n"
                    b"1 8 123456789\n2 2 0\n2 3 +7\n"),
    "slow_path_values": (b"2 9\n1 1 0.1234567890123456789012\n1 2 1e-300\n1 3 123456789012345678901234\n"
                         b"1 4 9007199254740993\n1 5 2.2250738585072014e-308\n1 6 1.7976931348623157e308\n"
                         b"1 7 4.9e-324\n1 8 3.14159265358979323846264338327950288\n"),
    "header_only": b"4 10\n",
    "unsorted_order5": b"5 20\n20 1 19 2 18 0.25\n3 3 1 3 2 -1.75\n",
}

MALFORMED = {
    "bad_value": b"3 6\n1 2 3 1.5x\n3 2 1 2\n",
    "bad_id": b"3 6\n1 2.5 3 1.5\n",
    "inf_value": b"2 4\n1 2 inf\n",
}


def random_text(seed: int, order: int = 4, dim: int = 5000, nnz: int = 100_000) -> bytes:
    """A large seeded file with mixed whitespace and value spellings."""
    rng = np.random.default_rng(seed)
    ids = rng.integers(1, dim + 1, size=(nnz, order))
    kind = rng.integers(0, 5, size=nnz)
    mant = rng.random(nnz)
    seps = [b" ", b"\t", b"  "]
    out = [f"{order} {dim}\n".encode()]
    for k in range(nnz):
        if kind[k] == 0:
            v = b"1"
        elif kind[k] == 1:
            v = f"{mant[k]:.6f}".encode()
        elif kind[k] == 2:
            v = f"{mant[k]:.17g}".encode()
        elif kind[k] == 3:
            v = f"{mant[k] * 10.0 ** int(rng.integers(-40, 40)):.9e}".encode()
        else:
            v = f"{-mant[k]:.3f}".encode()
        sep = seps[k % 3]
        out.append(sep.join([str(int(x)).encode() for x in ids[k]] + [v]) + (b"\r\n" if k % 7 == 0 else b"\n"))
    return b"".join(out)
