"""FP64 CPU restatement of the learned resize-factor network (test infrastructure only).

The network of srw_b200/learned.py: dense layers W (in x out) + b, GELU (tanh form, Hendrycks &
Gimpel 2016) between layers, identity on the last one, mean-squared-error loss.  Forward and
backward in numpy float64; ``numeric_grad`` checks the analytic gradients by central
differences.  Nothing in the product imports this module; the GPU tests compare the CUDA kernels'
results with it.  The network has no counterpart in the reference (its users choose the resize
factors by hand)."""
import numpy as np

C_GELU = 0.7978845608028654      # sqrt(2 / pi)


def gelu(z):
    return 0.5 * z * (1. + np.tanh(C_GELU * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(C_GELU * (z + 0.044715 * z ** 3))
    return 0.5 * (1. + t) + 0.5 * z * (1. - t * t) * C_GELU * (1. + 3. * 0.044715 * z * z)


def forward(X, Ws, bs):
    """Returns (output, pre-activations Z, activations Y with Y[0] = X)."""
    Y, Z = [np.asarray(X, np.float64)], []
    a = Y[0]
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = a @ np.asarray(W, np.float64) + np.asarray(b, np.float64)
        Z.append(z)
        a = gelu(z) if l + 1 < len(Ws) else z
        Y.append(a)
    return a, Z, Y


def mse(out, T):
    d = out - T
    return float(np.mean(d * d)), 2. * d / d.size


def backward(dOut, Ws, Z, Y):
    """dW, db of every layer given dLoss/dOut."""
    dW, db = [None] * len(Ws), [None] * len(Ws)
    d = np.asarray(dOut, np.float64)
    for l in range(len(Ws) - 1, -1, -1):
        if l + 1 < len(Ws):
            d = d * gelu_grad(Z[l])
        dW[l] = Y[l].T @ d
        db[l] = d.sum(0)
        if l > 0:
            d = d @ np.asarray(Ws[l], np.float64).T
    return dW, db


def numeric_grad(X, T, Ws, bs, l, idx, h=1e-6):
    """Central difference of the MSE loss with respect to W[l][idx]."""
    Wp = [np.array(w, np.float64) for w in Ws]
    Wm = [np.array(w, np.float64) for w in Ws]
    Wp[l][idx] += h
    Wm[l][idx] -= h
    lp = mse(forward(X, Wp, bs)[0], T)[0]
    lm = mse(forward(X, Wm, bs)[0], T)[0]
    return (lp - lm) / (2. * h)


def downsample64(I):
    """Mean of I over 64 x 64 cells, cell (cy, cx) = rows [cy ny/64, (cy+1) ny/64) x columns likewise."""
    ny, nx = I.shape
    out = np.zeros((64, 64))
    for cy in range(64):
        y0, y1 = cy * ny // 64, (cy + 1) * ny // 64
        for cx in range(64):
            x0, x1 = cx * nx // 64, (cx + 1) * nx // 64
            out[cy, cx] = I[y0:y1, x0:x1].mean() if (y1 > y0 and x1 > x0) else 0.
    return out
