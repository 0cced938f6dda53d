"""The statements the code generator emits for rate-coded learning (the
global, semiglobal and local equations with their bounds, the plasticity
switch and the period/offset test of proj<k>_update), compiled with g++ in
the update kernel's loop order around a plain C++ step of the learning case,
give the reference's own results bit for bit
(tests/golden/rate_learning.npz)."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest
import scipy.sparse as sp

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import learning_inputs  # noqa: E402
from test_zz_gpu_rate_learning import GOLD, build  # noqa: E402


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_generated_learning_statements_equal_reference(tmp_path):
    from annarchy_b200.core.backend import CompiledNetwork
    from annarchy_b200.generator.codegen import CodeGenerator
    net, inp, out, p1, p2, m, r_in = build("double")
    be = CompiledNetwork(net, dry=True)
    be.build()
    src = "".join(s for s, _ in CodeGenerator(be).rate_update_kernels(p1))

    def body(start, end):
        i = src.index(start)
        return src[i + len(start):src.index(end, i)]

    glob = body("if (anb_go && threadIdx.x == 0) {", "anb_p_proj0__beta[0] = beta;")
    glob = glob[glob.index("double _beta"):]
    semi = body("if (anb_lane == 0) {", "__syncwarp();").strip().rstrip("}")
    loc = body("j += 32) {", "__syncwarp();").strip().rstrip("}")
    r_in, W = learning_inputs()
    m1 = sp.csr_matrix(W)
    m1.sort_indices()
    rows = np.nonzero(np.diff(m1.indptr) > 0)[0]
    rp = np.concatenate([[0], np.cumsum(np.diff(m1.indptr)[rows])])
    arr = lambda a, t: "{" + ",".join(repr(float(x)) if t == "d" else str(int(x)) for x in a) + "}"
    out_bin = str(tmp_path / "out.bin")
    cpp = f"""
    #include <cstdio>
    #include <cmath>
    template <typename T> T positive(T x) {{ return x > T(0) ? x : T(0); }}
    const int NR = {len(rows)}, NNZ = {m1.nnz}, NIN = {len(r_in)}, NOUT = {W.shape[0]};
    int rows_[] = {arr(rows, 'i')}; int rp_[] = {arr(rp, 'i')}; int col_[] = {arr(m1.indices, 'i')};
    double w0[] = {arr(m1.data, 'd')}; double rin[] = {arr(r_in, 'd')};
    struct P {{ double w[NNZ]; double alpha[NR]; double beta = 1.0; double eta = 0.02, tau_alpha = 20.0;
               int fl[4] = {{1, 1, 1, 0}}; }};
    void upd(P& p, long long t, const double* anb_pre_r, const double* anb_post_r, double dt) {{
      const int anb_plastic = p.fl[0];
      if (!(p.fl[1] && (t - p.fl[3]) % p.fl[2] == 0)) return;
      const double anb_dt = dt * p.fl[2];
      {{ double& beta = p.beta; const double eta = p.eta, tau_alpha = p.tau_alpha; {glob} }}
      const double eta = p.eta, tau_alpha = p.tau_alpha, beta = p.beta;
      double* alpha = p.alpha; double* w = p.w; const int* anb_col = col_;
      for (int anb_row = 0; anb_row < NR; ++anb_row) {{
        const int anb_post = rows_[anb_row];
        {{ {semi} }}
        for (int j = rp_[anb_row]; j < rp_[anb_row + 1]; ++j) {{ {loc} }}
      }}
    }}
    int main() {{
      static P p1, p2;
      for (int j = 0; j < NNZ; ++j) {{ p1.w[j] = w0[j]; p2.w[j] = w0[j] * 0.5; }}
      for (int i = 0; i < NR; ++i) {{ p1.alpha[i] = 0; p2.alpha[i] = 0; }}
      double r[NOUT] = {{0}};
      FILE* f = fopen("{out_bin}", "wb");
      for (long long t = 0; t < 200; ++t) {{
        if (t == 7) {{ p2.fl[2] = 3; p2.fl[3] = 1; }}
        double se[NOUT] = {{0}}, sm[NOUT] = {{0}};
        for (int i = 0; i < NR; ++i) {{ double s = 0.0, q = 0.0;
          for (int j = rp_[i]; j < rp_[i + 1]; ++j) {{ s += rin[col_[j]] * p1.w[j]; q += rin[col_[j]] * p2.w[j]; }}
          se[rows_[i]] = 0.0 + s; sm[rows_[i]] = 0.0 + q; }}
        for (int i = 0; i < NOUT; ++i) {{ double _r = (se[i] + sm[i] - r[i]) / 10.0; r[i] += 1.0 * _r; }}
        upd(p1, t, rin, r, 1.0); upd(p2, t, rin, r, 1.0);
        fwrite(r, sizeof(double), NOUT, f);
      }}
      fwrite(p1.w, sizeof(double), NNZ, f); fwrite(p2.w, sizeof(double), NNZ, f);
      fwrite(p1.alpha, sizeof(double), NR, f); fwrite(p2.alpha, sizeof(double), NR, f);
      fwrite(&p1.beta, sizeof(double), 1, f); fwrite(&p2.beta, sizeof(double), 1, f);
      fclose(f); return 0;
    }}
    """
    (tmp_path / "harness.cpp").write_text(cpp)
    exe = str(tmp_path / "harness")
    subprocess.check_call(["g++", "-O2", "-ffp-contract=off", "-o", exe, str(tmp_path / "harness.cpp")])
    subprocess.check_call([exe])
    d = np.fromfile(out_bin, dtype=np.float64)
    n_out, nnz, nr = W.shape[0], m1.nnz, len(rows)
    sizes = [200 * n_out, nnz, nnz, nr, nr, 1, 1]
    parts = np.split(d, np.cumsum(sizes)[:-1])
    got = dict(r=parts[0].reshape(200, -1), w1=parts[1], w2=parts[2], alpha1=parts[3],
               alpha2=parts[4], beta1=parts[5][0], beta2=parts[6][0])
    for k, v in got.items():
        np.testing.assert_array_equal(np.asarray(v), GOLD[k], err_msg=k)
