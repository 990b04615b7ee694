"""The C++ layer include/lsmoke_gpu.hpp, which mirrors the reference's per-cell calls
(BatchReactorHomogeneousConstantPressure + MultiValueSolver, chemistry_DI.H:131-167) over a whole field.
A small program is compiled with g++ against the header and the library; on the CPU its error behaviour is
checked, on the GPU its results against the ctypes binding of the same C ABI."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "laminarsmoke_b200")

PROGRAM = r"""
#include "lsmoke_gpu.hpp"
#include <cstdio>
#include <fstream>
#include <vector>

int main(int argc, char** argv) {
  // error behaviour that needs no device
  if (lsmoke::ODE_STATUS_CONTINUATION != 2 || lsmoke::ODE_STATUS_MAX_NUMBER_CONVERGENCETEST_FAILURES != -5) return 10;
  lsmoke::BatchReactorHomogeneousConstantPressure reactor;
  try { reactor.SetReactor(-1.); return 11; } catch (const lsmoke::Error& e) { if (e.code() != LSG_ERR_ARG) return 12; }
  const char bad[16] = "NOTAMECHANISM00";
  try { lsmoke::Mechanism m(lsmoke::Blob{bad, 16}); return 13; } catch (const lsmoke::Error& e) { if (e.code() != LSG_ERR_MECH) return 14; }
  // the DRG settings (chemistry_DRG.H), set on the reactor as the reference does
  try { lsmoke::DRG none(std::vector<int>{}); return 17; } catch (const lsmoke::Error& e) { if (e.code() != LSG_ERR_ARG) return 18; }
  lsmoke::DRG drg({0, 1});
  try { drg.SetTemperatureBands({1000.}, {1e-2, 1e-3}); return 19; } catch (const lsmoke::Error& e) { if (e.code() != LSG_ERR_ARG) return 20; }
  drg.SetTemperatureBands({1200., 1e6}, {1e-3, 1e-2});
  if (drg.options().nbands != 2 || drg.options().nkey != 2 || drg.options().first_cell_options_only != 1) return 21;
  reactor.SetDRG(&drg);
  if (reactor.drg() != &drg) return 22;
  reactor.SetDRG(nullptr);
  if (argc < 5) {
    // the property map's interface compiles against the same header (its C entry point is tested on the GPU)
    void (lsmoke::TransportPropertiesMap::*ev)(int, const double*, const double*, const double*,
                                               lsmoke::TransportPropertiesMap::Fields&, double) =
        &lsmoke::TransportPropertiesMap::Evaluate;
    (void)ev;
    std::printf("cpu ok\n");
    return 0;
  }
  // the reference's call sequence on a field read from argv[2] (ncells, then Y[NC][ncells], then T[ncells])
  lsmoke::Mechanism mech(argv[1]);
  const int nc = mech.NumberOfSpecies();
  std::ifstream in(argv[2], std::ios::binary);
  int n = 0;
  in.read((char*)&n, sizeof(int));
  std::vector<double> Y((size_t)nc * n), T(n);
  in.read((char*)Y.data(), sizeof(double) * Y.size());
  in.read((char*)T.data(), sizeof(double) * T.size());
  std::vector<double*> Yp(nc);
  for (int i = 0; i < nc; ++i) Yp[i] = Y.data() + (size_t)i * n;
  reactor.SetReactor(101325.);
  reactor.SetEnergyEquation(true);
  lsmoke::MultiValueSolver solver(mech, reactor);
  std::vector<double> yMin(nc + 1, 0.), yMax(nc + 1, 1.);
  yMin[nc] = 200.;
  yMax[nc] = 6000.;
  solver.SetInitialConditions(0., n, Yp.data(), T.data());
  solver.SetFullPivoting(false);
  try { solver.SetFullPivoting(true); return 15; } catch (const lsmoke::Error& e) { if (e.code() != LSG_ERR_UNSUPPORTED) return 16; }
  solver.SetAbsoluteTolerances(std::atof(argv[4]) * 1e-5);
  solver.SetRelativeTolerances(std::atof(argv[4]));
  solver.SetMinimumValues(yMin);
  solver.SetMaximumValues(yMax);
  const std::vector<int>& st = solver.Solve(0. + 1e-5);
  std::ofstream out(argv[3], std::ios::binary);
  out.write((const char*)Y.data(), sizeof(double) * Y.size());
  out.write((const char*)T.data(), sizeof(double) * T.size());
  out.write((const char*)solver.QR().data(), sizeof(double) * n);
  out.write((const char*)st.data(), sizeof(int) * n);
  std::printf("gpu ok\n");
  return 0;
}
"""


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    lib = os.path.join(PKG, "liblsmoke_gpu.so")
    if not os.path.exists(lib):
        from laminarsmoke_b200.csrc import build
        build.build()
    src = tmp_path / "mirror.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "mirror"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", PKG, "-llsmoke_gpu", f"-Wl,-rpath,{PKG}"],
                   check=True, capture_output=True, text=True, timeout=300)
    return exe


def test_cpp_layer_compiles_and_reports_errors(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "cpu ok" in r.stdout


@pytest.mark.gpu
def test_cpp_layer_matches_the_c_abi(tmp_path, h2co, cuda):
    """The reference's call sequence through the C++ layer gives the ctypes step's result, bit for bit."""
    from laminarsmoke_b200 import cells, lsg
    from laminarsmoke_b200.mech import DATA
    _, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 256, seed=17)
    Ys = np.ascontiguousarray(Y.T)
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(np.int32(256).tobytes())
        f.write(Ys.tobytes())
        f.write(T.tobytes())
    exe = _build(tmp_path)
    rtol = 1e-7
    r = subprocess.run([str(exe), os.path.join(DATA, "POLIMI_H2CO_1412.lsmech"), str(tmp_path / "in.bin"),
                        str(tmp_path / "out.bin"), str(rtol)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    raw = (tmp_path / "out.bin").read_bytes()
    nc = len(species)
    Yc = np.frombuffer(raw, np.float64, nc * 256).reshape(nc, 256)
    Tc = np.frombuffer(raw, np.float64, 256, 8 * nc * 256)
    Qc = np.frombuffer(raw, np.float64, 256, 8 * (nc + 1) * 256)
    sc = np.frombuffer(raw, np.int32, 256, 8 * (nc + 2) * 256)
    ctx = lsg.ReactionStep(lsg.Mechanism(h2co[0]), rtol=rtol, atol=rtol * 1e-5)
    Yp = np.ascontiguousarray(Y.T)
    Tp = T.copy()
    Q, st, _ = ctx.step(Yp, Tp, 1e-5)
    np.testing.assert_array_equal(sc, st)
    np.testing.assert_array_equal(Yc, Yp)
    np.testing.assert_array_equal(Tc, Tp)
    np.testing.assert_array_equal(Qc, Q)
