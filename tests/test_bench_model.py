"""The algorithmic byte model behind bench.py's roofline line (no GPU).

Counts per map, in units of N^2 bytes, for float32 state and two components
(Q, U), n = 7 RK4 steps:
  forward row passes: init 12C, stage 1 (20C + 8), stages 2-4 (24C + 8), the last
  stage writes the output instead of y0 and S (-4C);
  adjoint row passes: init 16C + 8, stage 1 (24C + 8), stages 2-4 (28C + 8), last -8C;
  column passes 8C per stage; p planes 20 + 8 (2n + 1).
"""
import bench

P = 512 * 512


def test_forward_row_bytes():
    C, n = 2, 7
    expect = 12 * C + n * ((20 * C + 8) + 3 * (24 * C + 8)) - 4 * C
    assert bench.row_bytes_per_lens(C, n, P) == expect * P == 1528 * P


def test_adjoint_row_bytes():
    C, n = 2, 7
    expect = 16 * C + 8 + n * ((24 * C + 8) + 3 * (28 * C + 8)) - 8 * C
    assert bench.row_bytes_per_lens(C, n, P, adjoint=True) == expect * P == 1760 * P


def test_five_plane_path_reads_five_phi_planes_per_stage():
    C, n = 1, 7
    two = bench.row_bytes_per_lens(C, n, P, p_planes=2)
    five = bench.row_bytes_per_lens(C, n, P, p_planes=5)
    assert five - two == 4 * n * 12 * P  # three more float planes in each of the 4n stages


def test_column_and_p_plane_bytes():
    assert bench.col_bytes_per_lens(2, 7, P) == 28 * 16 * P
    assert bench.p_plane_bytes_per_lens(7, P) == (20 + 8 * 15) * P


def test_fused_phi_precompute_saves_the_plane_round_trip():
    # the derivative planes (20 N^2 written, 20 N^2 read back) no longer cross HBM on the p-plane path, and
    # the five derivative spectra cross it as float32 (20 N^2 written and read instead of 40)
    n = 7
    assert bench.phi_pp_bytes_per_map(n, P) == (80 + 8 * 15) * P
    assert 140 * P + bench.p_plane_bytes_per_lens(n, P) - bench.phi_pp_bytes_per_map(n, P) == 80 * P


def test_stage1_bytes_match_the_stage_model():
    # the launch whose DRAM traffic the roofline line reports
    assert bench.stage1_bytes_per_map(2) == 48
    assert bench.stage1_bytes_per_map(2, adjoint=True) == 56
    assert ("k_row_pair", 512, 2) in bench.NCU_STAGE1_TRAFFIC_PER_MAP
    assert ("k_row_pair_adj", 512, 2) in bench.NCU_STAGE1_TRAFFIC_PER_MAP
    for (name, n, c), per_map in bench.NCU_STAGE1_TRAFFIC_PER_MAP.items():
        # measured DRAM bytes: the reads (32 N^2) always, writes at most the algorithmic ones
        alg = bench.stage1_bytes_per_map(c, name.endswith("_adj")) * n * n
        assert 32 * n * n <= per_map * 1.001 and per_map <= alg


def test_workload_names():
    class A:
        adjoint, ncomp, nside, batch, nsteps, theta, gpus = False, 2, 512, 64, 7, 2.0, 1
    assert bench.workload_config(A)["workload"] == "lenseflow_fwd_qu512_b64_n7"
    A.adjoint = True
    assert bench.workload_config(A)["workload"] == "lenseflow_adj_qu512_b64_n7"
    assert bench.metric_name(A) == bench.METRIC_ADJ


def test_per_map_totals_for_the_headline_workload():
    # 512^2 QU, n = 7, new phi per map: the totals the design notes quote (MB = 1e6 bytes)
    n, C = 7, 2
    rows = bench.row_bytes_per_lens(C, n, P)
    cols = bench.col_bytes_per_lens(C, n, P)
    phi = bench.phi_pp_bytes_per_map(n, P)
    assert round(rows / 1e6, 1) == 400.6
    assert round(cols / 1e6, 1) == 117.4
    assert round(phi / 1e6, 1) == 52.4
    assert round((rows + cols + phi) / 1e6, 1) == 570.4
    assert round(bench.survey_bytes_per_map(C, n, P) / 1e6, 1) == 716.2
