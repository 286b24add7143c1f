"""CPU oracle of the learned free-surface preconditioner (test infrastructure
only: tests import it to check the CUDA network's forward pass, loss and
parameter gradient).  There is no reference counterpart: the reference solves
the free surface with FMG / SRJ (src/lin_solve.f90) and preconditions nothing,
so this restates the network the CUDA kernels define:

  nodes : the slots of [0, n]^2 of each lozenge that are their own ghost
          source (lozenge, row j, column i order);
  taps  : the node and its neighbours (+1,0), (+1,+1), (0,+1), (-1,0),
          (-1,-1), (0,-1), resolved through the ghost remap; -1 outside;
  net   : x = [r / rms(r), (r / rms(r)) (|H| / 2750 - 1)] -> 32 -> 32 -> 1
          channels, each a 7-tap convolution with BF16-rounded weights, no
          biases; the two hidden layers end in act(p) = p (p > 0), slope p
          (p <= 0) and are stored rounded to BF16 (the next layer reads the
          rounded values; the gradient passes straight through the rounding,
          and act' is taken from the sign of the stored value);
  use   : z = rms(r) y own, own = 0 at the pole slots (slots outside
          [0, n)^2) and 1 elsewhere; the solver adds it to a V-cycle's
          correction, z = c + net(r - L c);
  loss  : <d, -L d>_W / |W| with d = own y - e / rms(r), W the cell areas
          1 / hex_inv (the error in the energy norm of the solve).

Everything is evaluated in float64 from BF16/float32-rounded values, so the
CUDA results differ by FP32 accumulation order (and, rarely, by one BF16
rounding step of a hidden activation that this order moves across a rounding
boundary)."""
import numpy as np

TAPS, C, CIN = 7, 32, 2
DI = (0, 1, 1, 0, -1, -1, 0)
DJ = (0, 0, 1, 1, 0, -1, -1)
SHAPES = [("W1", (TAPS, CIN, C)), ("W2", (TAPS, C, C)), ("W3", (TAPS, C, 1))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16_round(w):
    """Round float32 values to the nearest BF16 value (ties to even), as float32."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(theta):
    out, o = {}, 0
    for name, shp in SHAPES:
        k = int(np.prod(shp))
        out[name] = np.asarray(theta[o:o + k], dtype=np.float64).reshape(shp)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def node_src(lv):
    """Ghost remap of a level: nsrc[k] = source slot of slot k."""
    from .grid import own
    lv = own(lv)
    nsrc = np.arange(lv.NN)
    nsrc[lv.halo_node[:, 0]] = lv.halo_node[:, 1]
    return nsrc


def layout(lv):
    """(slot, tap): the node slots (ns,) and the taps (7, ns) of one level."""
    n, P = lv.n, lv.P
    nsrc = node_src(lv)
    d, j, i = np.meshgrid(np.arange(10), np.arange(n + 1), np.arange(n + 1), indexing="ij")
    k = ((d * P + j + 2) * P + i + 2).ravel()
    slot = k[nsrc[k] == k]
    cid = np.full(lv.NN, -1, dtype=np.int64)
    cid[slot] = np.arange(slot.size)
    dd, rr = slot // (P * P), slot % (P * P)
    ii, jj = rr % P - 2, rr // P - 2
    tap = np.stack([cid[nsrc[(dd * P + jj + DJ[t] + 2) * P + ii + DI[t] + 2]] for t in range(TAPS)])
    return slot, tap


def _gather(a, tap_t):
    g = np.zeros((a.shape[0], tap_t.size))
    ok = tap_t >= 0
    g[:, ok] = a[:, tap_t[ok]]
    return g


def _conv(a, W, tap):
    out = np.zeros((W.shape[2], a.shape[1]))
    for t in range(TAPS):
        out += W[t].T @ _gather(a, tap[t])
    return out


def act(p, slope):
    return np.where(p > 0, p, slope * p)


def dact(h, slope):
    """act' from the stored output h (its sign is its argument's)."""
    return np.where(h > 0, 1.0, slope)


def _store(h):
    """A hidden activation as the kernels store it: FP32, then BF16."""
    return bf16_round(h.astype(np.float32)).astype(np.float64)


def forward(theta, r, depth, tap, round_weights=True, slope=1.0):
    """Activations of the network for compact residual r and depth |H| (ns,);
    round_weights=False leaves the weights and the hidden activations
    unrounded.  Returns a dict with x, h1, h2, y (channel-major), rs, slope and the
    parameters P used."""
    P = unpack(bf16_round(np.asarray(theta, np.float32)) if round_weights else theta)
    r = np.asarray(r, np.float64)
    rs = np.sqrt(np.mean(r * r))
    if not rs > 0:
        rs = 1.0
    v = (r / rs).astype(np.float32)
    x = np.stack([v, v * (np.abs(depth) / 2750.0 - 1.0).astype(np.float32)]).astype(np.float64)
    st = _store if round_weights else (lambda h: h)    # unrounded: the exact network, for finite differences
    h1 = st(act(_conv(x, P["W1"], tap), slope))
    h2 = st(act(_conv(h1, P["W2"], tap), slope))
    y = _conv(h2, P["W3"], tap)[0]
    return {"x": x, "h1": h1, "h2": h2, "y": y, "rs": rs, "P": P, "slope": slope}


def _conv_back(a, W, dout, tap):
    """Gradients of one layer: (dW, din) for input a and output gradient dout."""
    dW = np.zeros_like(W)
    din = np.zeros_like(a)
    for t in range(TAPS):
        g = _gather(a, tap[t])
        dW[t] = g @ dout.T
        contrib = W[t] @ dout
        ok = tap[t] >= 0
        np.add.at(din.T, tap[t][ok], contrib[:, ok].T)
    return dW, din


def backward(A, dy, tap):
    """Parameter gradient of the network from the output gradient dy (ns,),
    straight through the BF16 roundings (of the weights and the stored
    activations)."""
    dy = np.asarray(dy, np.float64)[None, :]
    P, slope = A["P"], A["slope"]
    dW3, dh2 = _conv_back(A["h2"], P["W3"], dy, tap)
    dW2, dh1 = _conv_back(A["h1"], P["W2"], dh2 * dact(A["h2"], slope), tap)
    dW1, _ = _conv_back(A["x"], P["W1"], dh1 * dact(A["h1"], slope), tap)
    return pack({"W1": dW1, "W2": dW2, "W3": dW3})


def loss_and_grad(theta, r, e, depth, tap, round_weights=True, slope=1.0):
    """Mean-square head (1/ns) sum (y - e/rs)^2 and its exact gradient: pins
    the network's backward pass against finite differences."""
    A = forward(theta, r, depth, tap, round_weights, slope)
    d = A["y"] - np.asarray(e, np.float64) / A["rs"]
    return float(np.mean(d * d)), backward(A, 2.0 * d / d.size, tap)


def energy_loss_and_grad(theta, r, e, depth, tap, slot, hinv, NN, apply_L, own, slope=1.0):
    """The training loss of the CUDA network: the error in the energy norm,
      loss = <d, -L d>_W / |W|,  d = own y - e/rs,  W = 1/hex_inv on the nodes,
    with apply_L(q) = L q for a level array q (ghosts not filled), and the
    gradient the CUDA kernels use, dy = 2 W (-L d) / |W| (exact when L is
    self-adjoint in <,>_W; the discrete operator is, to a few tenths of a
    percent)."""
    A = forward(theta, r, depth, tap, slope=slope)
    d = np.zeros(NN)
    d[slot] = own * A["y"] - np.asarray(e, np.float64) / A["rs"]
    w = 1.0 / np.asarray(hinv, np.float64)[slot]
    inv_area = 1.0 / w.sum()
    a = -apply_L(d)[slot] * w
    loss = float((d[slot] * a).sum() * inv_area)
    return loss, backward(A, own * 2.0 * a * inv_area, tap)


def infer(theta, r, depth, tap, own, slope=1.0):
    """The network's correction z = rs * y * own."""
    A = forward(theta, r, depth, tap, slope=slope)
    return A["rs"] * A["y"] * own


def init_params(seed):
    """Random parameters with the CUDA set-up's scales (variance-preserving
    linear layers, a small last layer; not the same random stream)."""
    rng = np.random.default_rng(seed)
    d = {"W1": rng.standard_normal((TAPS, CIN, C)) * np.sqrt(1.0 / (TAPS * CIN)),
         "W2": rng.standard_normal((TAPS, C, C)) * np.sqrt(1.0 / (TAPS * C)),
         "W3": rng.standard_normal((TAPS, C, 1)) * 0.1 * np.sqrt(1.0 / (TAPS * C))}
    return pack(d).astype(np.float32)
