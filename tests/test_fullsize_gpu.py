"""Size-independent properties of the BSIM4 load at the benchmark's full size (~1M instances),
where the oracle cannot follow in seconds: every instance's terminal currents and charges sum to
zero (KCL, charge conservation), its 4x4 dF/dx and dQ/dx blocks have zero row and column sums
(a common shift of all terminal voltages changes nothing; what leaves one terminal enters
another), and repeated loads are bit-identical."""
import numpy as np
import pytest

from xyce_b200 import Bsim4Device, SolverFlags, netlist

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tests.parity import family_inputs  # noqa: E402


@pytest.fixture(scope="module")
def full():
    c = netlist.random_logic(1_000_000, seed=2026, wire_segments=1)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c)
    dev = Bsim4Device(cards, im, nd, params, (rowptr, colind), c.n_unknowns)
    yield c, rowptr, dev
    dev.close()


def _load(dev, c, rowptr, sol, flags):
    n, nu, nnz = dev.n, c.n_unknowns, int(rowptr[-1])
    f64 = dict(dtype=torch.float64, device="cuda")
    sta, sto = torch.zeros(3 * n, **f64), torch.zeros(14 * n, **f64)
    out = [torch.zeros(nu, **f64) for _ in range(4)] + [torch.zeros(nnz, **f64) for _ in range(2)]
    dev.load(flags, torch.as_tensor(sol, **f64), sta, sta.clone(), sto, sto.clone(), *out)
    torch.cuda.synchronize()
    return out


def test_conservation_of_every_instance_at_full_size(full):
    c, rowptr, dev = full
    sol = np.random.default_rng(5).uniform(0.0, 1.2, c.n_unknowns)
    _load(dev, c, rowptr, sol, SolverFlags(newton_iter=1, voltlim=0))
    st = dev.copy_stamps()  # [48, n]
    F, Q = st[0:4], st[4:8]
    JF, JQ = st[16:32].reshape(4, 4, -1), st[32:48].reshape(4, 4, -1)
    tol = 1e-12
    for name, v in (("F", F), ("Q", Q)):
        scale = np.abs(v).sum(0) + 1e-300
        assert np.all(np.abs(v.sum(0)) <= tol * scale + 1e-30), name
    for name, J in (("dFdx", JF), ("dQdx", JQ)):
        scale = np.abs(J).sum((0, 1)) + 1e-300
        assert np.all(np.abs(J.sum(1)) <= 1e-11 * scale + 1e-30), name + " rows"
        assert np.all(np.abs(J.sum(0)) <= 1e-11 * scale + 1e-30), name + " columns"


def test_full_size_loads_are_bit_identical(full):
    c, rowptr, dev = full
    sol = np.random.default_rng(6).uniform(0.0, 1.2, c.n_unknowns)
    a = _load(dev, c, rowptr, sol, SolverFlags(newton_iter=1, voltlim=0))
    b = _load(dev, c, rowptr, sol, SolverFlags(newton_iter=1, voltlim=0))
    for x, y in zip(a, b):
        assert torch.equal(x, y)
