"""CPU oracle of the learned preconditioner (numpy) -- TEST INFRASTRUCTURE ONLY.

The network has no counterpart in qcu; this is an independent numpy
statement of the same mathematics, used to check the CUDA forward and
backward kernels.  Fields are complex128 arrays [B, 2, Vh, C, 3]
(parity-major, PyQuda even-odd site order, see oracle/qcu_oracle.c); one
parallel-transport layer computes

    out_a(x) = sum_{h=0..8} sum_b W[h, a, b] (T_h in_b)(x)

with T_0 = 1, T_{1+2mu} in(x) = U_mu(x) in(x+mu), T_{2+2mu} in(x) =
U_mu(x-mu)^dag in(x-mu), and the t-boundary phase on hops crossing t.
The network is N(r) = L2(L1(r)) with L1: 4 -> 16 channels (r on the odd
sites), L2: 16 -> 4 channels on the odd sites.  Weights are a float vector:
layer 1 [9,16,4] then layer 2 [9,4,16], complex as (re, im) pairs.
"""
import numpy as np

HOPS = 9
C_IN, C_HID, C_OUT = 4, 16, 4
N_W1 = HOPS * C_HID * C_IN
N_W2 = HOPS * C_OUT * C_HID


def split_weights(w):
    z = np.asarray(w, np.float64).reshape(-1, 2)
    z = z[:, 0] + 1j * z[:, 1]
    return z[:N_W1].reshape(HOPS, C_HID, C_IN), z[N_W1:].reshape(HOPS, C_OUT, C_HID)


def join_weights(w1, w2):
    z = np.concatenate([w1.ravel(), w2.ravel()])
    return np.stack([z.real, z.imag], axis=1).ravel()


class Lattice:
    """neighbour tables of the even-odd lattice and the links as 3x3 matrices"""

    def __init__(self, gauge, latt, t_bc=1.0):
        Lx, Ly, Lz, Lt = latt
        self.latt = latt
        self.Vh = Lx * Ly * Lz * Lt // 2
        Lxh = Lx // 2
        self.U = np.asarray(gauge).reshape(4, 2, self.Vh, 3, 3)
        i = np.arange(self.Vh)
        xh = i % Lxh
        y = (i // Lxh) % Ly
        z = (i // (Lxh * Ly)) % Lz
        t = i // (Lxh * Ly * Lz)
        self.fwd = np.zeros((4, 2, self.Vh), np.int64)
        self.bwd = np.zeros((4, 2, self.Vh), np.int64)
        self.ph_f = np.ones((4, 2, self.Vh))
        self.ph_b = np.ones((4, 2, self.Vh))
        L = [Lx, Ly, Lz, Lt]
        for p in (0, 1):
            x = 2 * xh + ((y + z + t + p) & 1)
            c = [x, y, z, t]
            for mu in range(4):
                for step, tab, ph in ((1, self.fwd, self.ph_f), (-1, self.bwd, self.ph_b)):
                    n = [v.copy() for v in c]
                    n[mu] = (c[mu] + step) % L[mu]
                    tab[mu, p] = ((n[3] * Lz + n[2]) * Ly + n[1]) * Lxh + n[0] // 2
                    if mu == 3:
                        cross = (c[3] == Lt - 1) if step > 0 else (c[3] == 0)
                        ph[mu, p] = np.where(cross, t_bc, 1.0)

    def transport(self, f, h, p):
        """(T_h f)(x) for all x of parity p; f: [B, 2, Vh, C, 3] -> [B, Vh, C, 3]"""
        if h == 0:
            return f[:, p]
        mu, fwd = (h - 1) // 2, (h % 2 == 1)
        if fwd:
            n = self.fwd[mu, p]
            U = self.U[mu, p]  # link at x
            v = np.einsum("sij,bscj->bsci", U, f[:, 1 - p][:, n])
            return v * self.ph_f[mu, p][None, :, None, None]
        n = self.bwd[mu, p]
        U = self.U[mu, 1 - p][n]  # link at x - mu
        v = np.einsum("sji,bscj->bsci", U.conj(), f[:, 1 - p][:, n])
        return v * self.ph_b[mu, p][None, :, None, None]


def bf16_round_complex(z):
    """real and imaginary parts rounded to bfloat16, as the tensor-core layer's A operand"""
    z = np.asarray(z, complex)
    return bf16_round(z.real.astype(np.float32)).astype(np.float64) + 1j * bf16_round(
        z.imag.astype(np.float32)).astype(np.float64)


def layer(lat, W, f, out_parities, round_act=False):
    """one parallel-transport layer; returns [B, 2, Vh, Cout, 3] (zero on other parities).
    round_act: the transported inputs rounded to bf16 before the channel
    mixing (the tensor-core layer, whose MMA operands are bf16)."""
    B = f.shape[0]
    out = np.zeros((B, 2, lat.Vh, W.shape[1], 3), complex)
    for p in out_parities:
        for h in range(HOPS):
            v = lat.transport(f, h, p)
            if round_act:
                v = bf16_round_complex(v)
            out[:, p] += np.einsum("ab,nsbx->nsax", W[h], v)
    return out


def forward(lat, w, r_odd, round_act=False):
    """N(r) for odd half spinors r [B, Vh, 4, 3] -> (output odd [B, Vh, 4, 3], hidden).
    round_act: the tensor-core network, whose MMA operands (the transported
    inputs) are bf16 and whose hidden field is stored as bf16."""
    w1, w2 = split_weights(w)
    B = r_odd.shape[0]
    f0 = np.zeros((B, 2, lat.Vh, C_IN, 3), complex)
    f0[:, 1] = r_odd
    hid = layer(lat, w1, f0, (0, 1), round_act)
    if round_act:
        hid = bf16_round_complex(hid)
    out = layer(lat, w2, hid, (1,), round_act)
    return out[:, 1], hid, f0


def loss(lat, w, r_odd, e_odd):
    o, _, _ = forward(lat, w, r_odd)
    en = np.sum(np.abs(e_odd) ** 2, axis=(1, 2, 3))
    return float(np.mean(np.sum(np.abs(o - e_odd) ** 2, axis=(1, 2, 3)) / en))


def wgrad(lat, W_shape_out, delta, f, out_parities):
    """G[h, a, b] = sum_x sum_colour delta_a(x) conj((T_h f_b)(x))"""
    G = np.zeros((HOPS,) + W_shape_out, complex)
    for p in out_parities:
        for h in range(HOPS):
            G[h] += np.einsum("nsax,nsbx->ab", delta[:, p], lat.transport(f, h, p).conj())
    return G


def adjoint_layer(lat, W, delta, out_parities):
    """input gradient: sum_h sum_a conj(W[h, a, b]) (T_h^dag delta_a), T_h^dag = T_hbar"""
    bar = [0, 2, 1, 4, 3, 6, 5, 8, 7]
    Wadj = np.stack([W[bar[h]].conj().T for h in range(HOPS)])
    return layer(lat, Wadj, delta, out_parities)


def gradient(lat, w, r_odd, e_odd):
    """dL/dW* (the conjugate Wirtinger derivative, the convention of the CUDA
    kernels) as a float vector in the weight layout, and the loss"""
    w1, w2 = split_weights(w)
    B = r_odd.shape[0]
    o, hid, f0 = forward(lat, w, r_odd)
    en = np.sum(np.abs(e_odd) ** 2, axis=(1, 2, 3))
    d2 = np.zeros((B, 2, lat.Vh, C_OUT, 3), complex)
    d2[:, 1] = (o - e_odd) / (en[:, None, None, None] * B)
    g2 = wgrad(lat, (C_OUT, C_HID), d2, hid, (1,))
    d1 = adjoint_layer(lat, w2, d2, (0, 1))
    g1 = wgrad(lat, (C_HID, C_IN), d1, f0, (0, 1))
    L = float(np.mean(np.sum(np.abs(o - e_odd) ** 2, axis=(1, 2, 3)) / en))
    return join_weights(g1, g2), L


def bf16_round(w):
    """round float32 values to bfloat16 (nearest-even), as the inference weights"""
    a = np.asarray(w, np.float32).view(np.uint32).astype(np.uint64)
    a = (a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000
    return a.astype(np.uint32).view(np.float32)
