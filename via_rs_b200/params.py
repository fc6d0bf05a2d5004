"""Parameter sets of the VIA answer path, as the C ABI's `via_params` struct.

Mirrors the reference's presets (crates/via-protocol/src/presets.rs:91-363) and
the parameter stacks its tests run end to end:

* ``toy_preset``   — TOY_PARAMS / ViaCToyParams (presets.rs:91,204-229):
  n1=64, n2=16, q1=2^40, q2=2^32, q3=2^16, q4=2^12, p=16, gadget bases 4/4/4,
  L_QUERY=20, L_CK=40, L_RSK=8. The preset does not fix the cascade base; it is
  2 here so that B^L_CK = 2^40 = q1, the same B^L = q pattern as its other
  gadgets.
* ``paper_preset`` — REALISTIC_PARAMS / ViaCRealisticParams (presets.rs:97,232-258)
  with the bases the paper-scale e2e test uses
  (crates/via-integration/tests/client_server_e2e_paper.rs:33-105).
* ``n8_preset``    — the n1=8 stack of crates/via-integration/tests/client_server_e2e.rs
  and layer6_kats.rs.
"""
import ctypes
import dataclasses

PAPER_Q1 = (137_438_822_401, 274_810_798_081)
PAPER_Q2 = 17_175_674_881
PAPER_Q3 = 8_380_417


class ViaParams(ctypes.Structure):
    """`via_params` from include/via_gpu.h (field order and types must match)."""

    _fields_ = [
        ("n1", ctypes.c_uint32),
        ("n2", ctypes.c_uint32),
        ("n_rec", ctypes.c_uint32),
        ("reserved0", ctypes.c_uint32),
        ("num_rows", ctypes.c_uint64),
        ("num_cols", ctypes.c_uint64),
        ("q1_0", ctypes.c_uint64),
        ("q1_1", ctypes.c_uint64),
        ("q2", ctypes.c_uint64),
        ("q3", ctypes.c_uint64),
        ("q4", ctypes.c_uint64),
        ("p", ctypes.c_uint64),
        ("b_dmux", ctypes.c_uint64),
        ("b_cmux", ctypes.c_uint64),
        ("ck_base", ctypes.c_uint64),
        ("b_rsk", ctypes.c_uint64),
        ("l_query", ctypes.c_uint32),
        ("l_ck", ctypes.c_uint32),
        ("l_rsk", ctypes.c_uint32),
        ("reserved1", ctypes.c_uint32),
    ]


@dataclasses.dataclass(frozen=True)
class Params:
    n1: int
    n2: int
    n_rec: int
    num_rows: int
    num_cols: int
    q1: tuple  # (q1_0, q1_1) for a two-prime RNS q1, (q1,) for a single modulus
    q2: int
    q3: int
    q4: int
    p: int
    b_dmux: int
    b_cmux: int
    ck_base: int
    b_rsk: int
    l_query: int
    l_ck: int
    l_rsk: int

    # ---- derived sizes (uint64 units, the include/via_gpu.h layouts) ----
    @property
    def nl(self) -> int:
        return len(self.q1)

    @property
    def d(self) -> int:
        return self.n1 // self.n2

    @property
    def q1_value(self) -> int:
        v = 1
        for q in self.q1:
            v *= q
        return v

    @property
    def num_dmux(self) -> int:
        return self.num_rows.bit_length() - 1

    @property
    def num_cmux(self) -> int:
        return self.num_cols.bit_length() - 1

    @property
    def num_crot(self) -> int:
        r = self.n1 // self.n_rec
        return r.bit_length() - 1 if r > 1 else 0

    @property
    def n_lwe(self) -> int:
        return (self.num_dmux + self.num_cmux + self.num_crot) * self.l_query

    @property
    def lwe_len(self) -> int:
        return self.nl * (self.n1 + 1)

    @property
    def cascade_key_len(self) -> int:
        steps = self.n1.bit_length() - 1
        return steps * (2 * self.n1) * self.l_ck * 2 * self.nl

    @property
    def conv_key_len(self) -> int:
        return self.l_ck * 2 * self.nl * self.n1

    @property
    def rsk_len(self) -> int:
        return self.d * self.l_rsk * 2 * self.n2

    @property
    def capacity(self) -> int:
        return self.num_rows * self.num_cols * (self.n1 // self.n_rec)

    def with_dims(self, num_rows: int, num_cols: int, n_rec: int | None = None) -> "Params":
        return dataclasses.replace(
            self, num_rows=num_rows, num_cols=num_cols, n_rec=self.n_rec if n_rec is None else n_rec
        )

    def to_c(self) -> ViaParams:
        c = ViaParams()
        c.n1, c.n2, c.n_rec = self.n1, self.n2, self.n_rec
        c.num_rows, c.num_cols = self.num_rows, self.num_cols
        c.q1_0 = self.q1[0]
        c.q1_1 = self.q1[1] if len(self.q1) > 1 else 0
        c.q2, c.q3, c.q4, c.p = self.q2, self.q3, self.q4, self.p
        c.b_dmux, c.b_cmux, c.ck_base, c.b_rsk = self.b_dmux, self.b_cmux, self.ck_base, self.b_rsk
        c.l_query, c.l_ck, c.l_rsk = self.l_query, self.l_ck, self.l_rsk
        return c


def paper_preset(num_rows: int = 256, num_cols: int = 4096, n_rec: int = 512) -> Params:
    """Paper VIA-C parameters; 1 GiB of 4-bit records at I=2^8, J=2^12."""
    return Params(
        n1=2048, n2=512, n_rec=n_rec, num_rows=num_rows, num_cols=num_cols,
        q1=PAPER_Q1, q2=PAPER_Q2, q3=PAPER_Q3, q4=4096, p=16,
        b_dmux=55879, b_cmux=81, ck_base=18, b_rsk=8,
        l_query=2, l_ck=18, l_rsk=8,
    )


SECURE_Q1 = (173_964_607_489, 173_964_656_641)


def secure_preset(num_rows: int = 256, num_cols: int = 4096, n_rec: int = 1024) -> Params:
    """SECURE_PARAMS (crates/via-protocol/src/presets.rs:278-303): the >= 120-bit
    VIA-C preset, n1=4096, n2=1024, q1 two 38-bit primes, q4=2^15, erratum gadgets."""
    return Params(
        n1=4096, n2=1024, n_rec=n_rec, num_rows=num_rows, num_cols=num_cols,
        q1=SECURE_Q1, q2=PAPER_Q2, q3=PAPER_Q3, q4=1 << 15, p=16,
        b_dmux=18073, b_cmux=307, ck_base=18, b_rsk=4,
        l_query=2, l_ck=18, l_rsk=8,
    )


def toy_preset(num_rows: int = 16, num_cols: int = 16, n_rec: int = 16) -> Params:
    """TOY_PARAMS; 1024 records of 16 4-bit coefficients at I=J=16."""
    return Params(
        n1=64, n2=16, n_rec=n_rec, num_rows=num_rows, num_cols=num_cols,
        q1=(1 << 40,), q2=1 << 32, q3=1 << 16, q4=1 << 12, p=16,
        b_dmux=4, b_cmux=4, ck_base=2, b_rsk=4,
        l_query=20, l_ck=40, l_rsk=8,
    )


def n8_preset(num_rows: int = 2, num_cols: int = 2) -> Params:
    """The n1=8 toy stack of the reference's client_server_e2e / layer6 KATs."""
    return Params(
        n1=8, n2=4, n_rec=4, num_rows=num_rows, num_cols=num_cols,
        q1=(1 << 36,), q2=1 << 28, q3=1 << 20, q4=1 << 12, p=16,
        b_dmux=64, b_cmux=64, ck_base=64, b_rsk=8,
        l_query=7, l_ck=7, l_rsk=8,
    )
