// PyTorch extension module `DTCSpMM`: the reference's Python-facing API
// (DTC-SpMM/DTCSpMM.cpp:361-399) over the C ABI of libdtcspmm.so.
//
// Same names, argument order and meaning as the reference. Differences, all
// deliberate: errors raise RuntimeError instead of exit(-1); each call runs
// its kernel once on the current stream (the reference launches 1000 times,
// appends a CSV row in the working directory and prints timing); optional
// keyword `values` carries real A values (the reference hard-codes A = 1).
#include <torch/extension.h>
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>
#include <string>
#include <tuple>
#include <vector>
#include "dtc_spmm.h"

namespace {

#define CHECK_DEV(x) TORCH_CHECK((x).is_cuda(), #x " must be a CUDA tensor")
#define CHECK_CONTIG(x) TORCH_CHECK((x).is_contiguous(), #x " must be contiguous")
#define CHECK_INPUT(x) CHECK_DEV(x); CHECK_CONTIG(x)
#define CHECK_DTYPE(x, t) TORCH_CHECK((x).scalar_type() == (t), #x " has the wrong dtype")

void check(dtc_status s, const char* what) {
  TORCH_CHECK(s == DTC_OK, what, " failed (status ", (int)s, "): ", dtc_last_error());
}

dtc_stream_t cur_stream() { return (dtc_stream_t)at::cuda::getCurrentCUDAStream().stream(); }

// DTCSpMM.cpp:313-359 preprocess_gpu. blockPartition / edgeToColumn /
// edgeToRow are written in place like the reference's; returns
// (RowWindowOffset, TCblockRowid, TCblocktileId, TCblockoffset, SparseAToX, T)
// and, when `values` (CSR order) is given, TCvalues (tile order) appended.
py::tuple preprocess_gpu(torch::Tensor edgeList, torch::Tensor nodePointer, int64_t num_nodes,
                         int64_t blockSize_h, int64_t blockSize_w, torch::Tensor blockPartition,
                         torch::Tensor edgeToColumn, torch::Tensor edgeToRow,
                         c10::optional<torch::Tensor> values) {
  CHECK_INPUT(edgeList); CHECK_INPUT(nodePointer); CHECK_INPUT(blockPartition);
  CHECK_INPUT(edgeToColumn); CHECK_INPUT(edgeToRow);
  CHECK_DTYPE(edgeList, torch::kInt32); CHECK_DTYPE(nodePointer, torch::kInt32);
  CHECK_DTYPE(blockPartition, torch::kInt32); CHECK_DTYPE(edgeToColumn, torch::kInt32);
  CHECK_DTYPE(edgeToRow, torch::kInt32);
  const c10::cuda::CUDAGuard guard(edgeList.device());
  const int64_t nnz = edgeList.numel();
  const int64_t nwin = (num_nodes + blockSize_h - 1) / blockSize_h;
  TORCH_CHECK(nodePointer.numel() == num_nodes + 1, "nodePointer must have num_nodes+1 entries");
  TORCH_CHECK(blockPartition.numel() >= nwin, "blockPartition needs ceil(num_nodes/blockSize_h) entries");
  TORCH_CHECK(edgeToColumn.numel() >= nnz && edgeToRow.numel() >= nnz, "edge arrays too small");
  auto i32 = torch::TensorOptions().dtype(torch::kInt32).device(edgeList.device());
  auto u8 = torch::TensorOptions().dtype(torch::kUInt8).device(edgeList.device());
  size_t wsb = 0;
  check(dtc_convert_workspace_bytes((int32_t)num_nodes, nnz, (int32_t)blockSize_h,
                                    (int32_t)blockSize_w, &wsb), "dtc_convert_workspace_bytes");
  auto ws = torch::empty({(int64_t)wsb}, u8);
  auto rwo = torch::zeros({nwin + 1}, i32);
  int64_t T = 0;
  check(dtc_convert_count(edgeList.data_ptr<int32_t>(), nodePointer.data_ptr<int32_t>(),
                          (int32_t)num_nodes, nnz, (int32_t)blockSize_h, (int32_t)blockSize_w,
                          blockPartition.data_ptr<int32_t>(), edgeToColumn.data_ptr<int32_t>(),
                          edgeToRow.data_ptr<int32_t>(), rwo.data_ptr<int32_t>(), ws.data_ptr(),
                          wsb, &T, cur_stream()), "dtc_convert_count");
  auto rowid = torch::zeros({T}, i32);
  auto tile = torch::zeros({nnz}, u8);
  auto toff = torch::zeros({T + 1}, i32);
  auto s2x = torch::zeros({T * blockSize_w}, i32);
  torch::Tensor tv;
  const float* vptr = nullptr;
  float* tvptr = nullptr;
  if (values.has_value()) {
    auto v = values.value();
    CHECK_INPUT(v); CHECK_DTYPE(v, torch::kFloat32);
    TORCH_CHECK(v.numel() == nnz, "values must have nnz entries");
    tv = torch::zeros({nnz}, v.options());
    vptr = v.data_ptr<float>();
    tvptr = tv.data_ptr<float>();
  }
  check(dtc_convert_fill(edgeList.data_ptr<int32_t>(), nodePointer.data_ptr<int32_t>(),
                         (int32_t)num_nodes, nnz, (int32_t)blockSize_h, (int32_t)blockSize_w,
                         edgeToColumn.data_ptr<int32_t>(), edgeToRow.data_ptr<int32_t>(),
                         rwo.data_ptr<int32_t>(), T, rowid.data_ptr<int32_t>(),
                         tile.data_ptr<uint8_t>(), toff.data_ptr<int32_t>(),
                         s2x.data_ptr<int32_t>(), vptr, tvptr, ws.data_ptr(), wsb, cur_stream()),
        "dtc_convert_fill");
  if (values.has_value()) return py::make_tuple(rwo, rowid, tile, toff, s2x, T, tv);
  return py::make_tuple(rwo, rowid, tile, toff, s2x, T);
}

void check_metcf(const torch::Tensor& X, const torch::Tensor& a, const torch::Tensor& tile,
                 const torch::Tensor& toff, const torch::Tensor& s2x) {
  CHECK_INPUT(X); CHECK_INPUT(a); CHECK_INPUT(tile); CHECK_INPUT(toff); CHECK_INPUT(s2x);
  CHECK_DTYPE(X, torch::kFloat32); CHECK_DTYPE(a, torch::kInt32);
  CHECK_DTYPE(tile, torch::kUInt8); CHECK_DTYPE(toff, torch::kInt32);
  CHECK_DTYPE(s2x, torch::kInt32);
  TORCH_CHECK(X.dim() == 2, "X must be 2-D [num_nodes, N]");
}

const float* values_ptr(const c10::optional<torch::Tensor>& values, int64_t nnz) {
  if (!values.has_value()) return nullptr;
  auto& v = values.value();
  CHECK_INPUT(v); CHECK_DTYPE(v, torch::kFloat32);
  TORCH_CHECK(v.numel() == nnz, "values must have one entry per TC-block nonzero");
  return v.data_ptr<float>();
}

// Plans the reference accepts (DTCSpMM_kernel.cu:840-930); all run the
// tcgen05 kernel here (vector width / N split are not parameters of it).
// "mma_sync" selects the legacy-ISA kernel.
bool legacy_plan(const std::string& plan) {
  static const char* ok[] = {"float_nonsplit", "float2_nonsplit", "float2_split",
                             "float4_nonsplit", "float4_split", "tcgen05"};
  if (plan == "mma_sync") return true;
  for (auto* p : ok)
    if (plan == p) return false;
  TORCH_CHECK(false, "Not supported exe plan: ", plan);
  return false;
}

// DTCSpMM.cpp:117-131 run_DTCSpMM (window-scheduled).
std::vector<torch::Tensor> run_DTCSpMM(torch::Tensor X, torch::Tensor RowWindowOffset,
                                       torch::Tensor TCblocktileId, torch::Tensor TCblockoffset,
                                       torch::Tensor SparseAToX, int64_t num_nodes,
                                       int64_t num_edges, std::string exeplan,
                                       c10::optional<torch::Tensor> values) {
  check_metcf(X, RowWindowOffset, TCblocktileId, TCblockoffset, SparseAToX);
  const c10::cuda::CUDAGuard guard(X.device());
  TORCH_CHECK(X.size(0) == num_nodes, "X must have num_nodes rows");
  const bool legacy = legacy_plan(exeplan);
  auto C = torch::empty_like(X);
  const int32_t nwin = (int32_t)RowWindowOffset.numel() - 1;
  const int64_t T = TCblockoffset.numel() - 1;
  const float* vp = values_ptr(values, TCblocktileId.numel());
  if (legacy) {
    check(dtc_spmm_mma_sync(RowWindowOffset.data_ptr<int32_t>(), TCblocktileId.data_ptr<uint8_t>(),
                            TCblockoffset.data_ptr<int32_t>(), SparseAToX.data_ptr<int32_t>(), vp,
                            (int32_t)num_nodes, nwin, X.data_ptr<float>(), (int32_t)X.size(1),
                            C.data_ptr<float>(), cur_stream()), "dtc_spmm_mma_sync");
  } else if (X.size(1) % 4 != 0) {
    check(dtc_spmm(RowWindowOffset.data_ptr<int32_t>(), TCblocktileId.data_ptr<uint8_t>(),
                   TCblockoffset.data_ptr<int32_t>(), SparseAToX.data_ptr<int32_t>(), vp,
                   (int32_t)num_nodes, nwin, T, X.data_ptr<float>(), (int32_t)X.size(1),
                   C.data_ptr<float>(), cur_stream()), "dtc_spmm");
  } else {
    // the window-scheduled product with the chunk queue in a torch workspace
    const int32_t N = (int32_t)X.size(1);
    size_t wsb = 0;
    check(dtc_spmm_ex_workspace_bytes((int32_t)num_nodes, T, N, 16, 0, 0, &wsb),
          "dtc_spmm_ex_workspace_bytes");
    auto ws = torch::empty({(int64_t)(wsb > 0 ? wsb : 1)}, X.options().dtype(torch::kUInt8));
    check(dtc_spmm_ex(RowWindowOffset.data_ptr<int32_t>(), TCblocktileId.data_ptr<uint8_t>(),
                      TCblockoffset.data_ptr<int32_t>(), SparseAToX.data_ptr<int32_t>(), vp,
                      (int32_t)num_nodes, nwin, T, 16, 8, DTC_B_F32, X.data_ptr<float>(), nullptr,
                      N, DTC_PREC_TF32, C.data_ptr<float>(), 0, 0, 0, ws.data_ptr(), wsb,
                      cur_stream()), "dtc_spmm_ex");
  }
  return {C};
}

// DTCSpMM.cpp:147-161 DTCSpMM_gcn (single launch, A = 1 unless `values`).
// Optional `bias` [N] and `relu` are fused into the store of C
// (C = act(A X + bias)), the GCN layer's epilogue.
std::vector<torch::Tensor> DTCSpMM_gcn(torch::Tensor X, torch::Tensor RowWindowOffset,
                                       torch::Tensor TCblocktileId, torch::Tensor TCblockoffset,
                                       torch::Tensor SparseAToX, int64_t num_nodes,
                                       int64_t num_edges, c10::optional<torch::Tensor> values,
                                       c10::optional<torch::Tensor> bias, bool relu) {
  if (!bias.has_value() && !relu)
    return run_DTCSpMM(X, RowWindowOffset, TCblocktileId, TCblockoffset, SparseAToX, num_nodes,
                       num_edges, "tcgen05", values);
  check_metcf(X, RowWindowOffset, TCblocktileId, TCblockoffset, SparseAToX);
  const c10::cuda::CUDAGuard guard(X.device());
  TORCH_CHECK(X.size(0) == num_nodes, "X must have num_nodes rows");
  const int32_t N = (int32_t)X.size(1);
  const float* bp = nullptr;
  if (bias.has_value()) {
    auto& b = bias.value();
    CHECK_INPUT(b); CHECK_DTYPE(b, torch::kFloat32);
    TORCH_CHECK(b.numel() == N, "bias must have N entries");
    bp = b.data_ptr<float>();
  }
  auto C = torch::empty_like(X);
  const int32_t nwin = (int32_t)RowWindowOffset.numel() - 1;
  const int64_t T = TCblockoffset.numel() - 1;
  size_t wsb = 0;
  check(dtc_spmm_ex_workspace_bytes((int32_t)num_nodes, T, N, 16, 0, 0, &wsb),
        "dtc_spmm_ex_workspace_bytes");
  auto ws = torch::empty({(int64_t)(wsb > 0 ? wsb : 1)}, X.options().dtype(torch::kUInt8));
  check(dtc_spmm_fused(RowWindowOffset.data_ptr<int32_t>(), TCblocktileId.data_ptr<uint8_t>(),
                       TCblockoffset.data_ptr<int32_t>(), SparseAToX.data_ptr<int32_t>(),
                       values_ptr(values, TCblocktileId.numel()), (int32_t)num_nodes, nwin, T, 16,
                       8, DTC_B_F32, X.data_ptr<float>(), nullptr, N, DTC_PREC_TF32, bp,
                       relu ? 1 : 0, C.data_ptr<float>(), 0, 0, 0, ws.data_ptr(), wsb,
                       cur_stream()),
        "dtc_spmm_fused");
  return {C};
}

// DTCSpMM.cpp:163-178 run_DTCSpMM_balance (strict balance, deterministic).
std::vector<torch::Tensor> run_DTCSpMM_balance(torch::Tensor X, torch::Tensor TCblockRowid,
                                               torch::Tensor TCblocktileId,
                                               torch::Tensor TCblockoffset,
                                               torch::Tensor SparseAToX, int64_t num_nodes,
                                               std::string exeplan,
                                               c10::optional<torch::Tensor> values) {
  check_metcf(X, TCblockRowid, TCblocktileId, TCblockoffset, SparseAToX);
  const c10::cuda::CUDAGuard guard(X.device());
  TORCH_CHECK(X.size(0) == num_nodes, "X must have num_nodes rows");
  TORCH_CHECK(exeplan == "float_nonsplit" || exeplan == "float4_split" || exeplan == "tcgen05",
              "Not supported exe plan: ", exeplan);
  auto C = torch::empty_like(X);
  const int64_t T = TCblockRowid.numel();
  const int32_t N = (int32_t)X.size(1);
  size_t wsb = 0;
  check(dtc_spmm_balance_workspace_bytes((int32_t)num_nodes, T, N, &wsb),
        "dtc_spmm_balance_workspace_bytes");
  auto ws = torch::empty({(int64_t)wsb}, X.options().dtype(torch::kUInt8));
  check(dtc_spmm_balance(TCblockRowid.data_ptr<int32_t>(), TCblocktileId.data_ptr<uint8_t>(),
                         TCblockoffset.data_ptr<int32_t>(), SparseAToX.data_ptr<int32_t>(),
                         values_ptr(values, TCblocktileId.numel()), (int32_t)num_nodes, T,
                         X.data_ptr<float>(), N, C.data_ptr<float>(), ws.data_ptr(), wsb,
                         cur_stream()), "dtc_spmm_balance");
  return {C};
}

// Extension beyond the reference: any B storage form / precision / schedule.
// Bplanes: [plane0, plane1?] produced by pack_b; mode 0 window, 1 balance.
std::vector<torch::Tensor> run_DTCSpMM_ex(std::vector<torch::Tensor> Bplanes, int64_t bformat,
                                          int64_t N, torch::Tensor RowWindowOffset,
                                          torch::Tensor TCblocktileId, torch::Tensor TCblockoffset,
                                          torch::Tensor SparseAToX, int64_t num_nodes,
                                          int64_t precision, int64_t mode, int64_t grid,
                                          c10::optional<torch::Tensor> values, int64_t ntile,
                                          int64_t block_h, int64_t block_w) {
  TORCH_CHECK(!Bplanes.empty(), "Bplanes is empty");
  for (auto& t : Bplanes) { CHECK_INPUT(t); }
  const c10::cuda::CUDAGuard guard(Bplanes[0].device());
  auto C = torch::empty({num_nodes, N}, Bplanes[0].options().dtype(torch::kFloat32));
  const int32_t nwin = (int32_t)RowWindowOffset.numel() - 1;
  const int64_t T = TCblockoffset.numel() - 1;
  size_t wsb = 0;
  check(dtc_spmm_ex_workspace_bytes((int32_t)num_nodes, T, (int32_t)N, (int32_t)block_h, (int)mode,
                                    (int)grid, &wsb),
        "dtc_spmm_ex_workspace_bytes");
  auto ws = torch::empty({(int64_t)(wsb > 0 ? wsb : 1)}, C.options().dtype(torch::kUInt8));
  check(dtc_spmm_ex(RowWindowOffset.data_ptr<int32_t>(), TCblocktileId.data_ptr<uint8_t>(),
                    TCblockoffset.data_ptr<int32_t>(), SparseAToX.data_ptr<int32_t>(),
                    values_ptr(values, TCblocktileId.numel()), (int32_t)num_nodes, nwin, T,
                    (int32_t)block_h, (int32_t)block_w, (int)bformat, Bplanes[0].data_ptr(),
                    Bplanes.size() > 1 ? Bplanes[1].data_ptr() : nullptr, (int32_t)N,
                    (int)precision, C.data_ptr<float>(), (int)mode, (int)grid, (int)ntile,
                    ws.data_ptr(), wsb, cur_stream()), "dtc_spmm_ex");
  return {C};
}

std::vector<torch::Tensor> pack_b(torch::Tensor B, int64_t bformat) {
  CHECK_INPUT(B); CHECK_DTYPE(B, torch::kFloat32);
  const c10::cuda::CUDAGuard guard(B.device());
  const int64_t rows = B.size(0), N = B.size(1);
  size_t b0 = 0, b1 = 0;
  check(dtc_bformat_bytes((int)bformat, rows, (int32_t)N, &b0, &b1), "dtc_bformat_bytes");
  auto p0 = torch::empty({(int64_t)b0}, B.options().dtype(torch::kUInt8));
  auto p1 = torch::empty({(int64_t)(b1 > 0 ? b1 : 1)}, B.options().dtype(torch::kUInt8));
  check(dtc_pack_b((int)bformat, B.data_ptr<float>(), rows, (int32_t)N, p0.data_ptr(),
                   b1 > 0 ? p1.data_ptr() : nullptr, cur_stream()), "dtc_pack_b");
  if (b1 > 0) return {p0, p1};
  return {p0};
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("preprocess_gpu", &preprocess_gpu, "ME-TCF conversion (CUDA)", py::arg("edgeList"),
        py::arg("nodePointer"), py::arg("num_nodes"), py::arg("blockSize_h"),
        py::arg("blockSize_w"), py::arg("blockPartition"), py::arg("edgeToColumn"),
        py::arg("edgeToRow"), py::arg("values") = py::none());
  m.def("run_DTCSpMM", &run_DTCSpMM, "DTC-SpMM forward, window-scheduled (CUDA)", py::arg("X"),
        py::arg("RowWindowOffset"), py::arg("TCblocktileId"), py::arg("TCblockoffset"),
        py::arg("SparseAToX"), py::arg("num_nodes"), py::arg("num_edges"), py::arg("exeplan"),
        py::arg("values") = py::none());
  m.def("run_DTCSpMM_balance", &run_DTCSpMM_balance, "DTC-SpMM strict-balance forward (CUDA)",
        py::arg("X"), py::arg("TCblockRowid"), py::arg("TCblocktileId"),
        py::arg("TCblockoffset"), py::arg("SparseAToX"), py::arg("num_nodes"),
        py::arg("exeplan"), py::arg("values") = py::none());
  m.def("DTCSpMM_gcn", &DTCSpMM_gcn, "DTC-SpMM forward for GCN, A = 1 (CUDA)", py::arg("X"),
        py::arg("RowWindowOffset"), py::arg("TCblocktileId"), py::arg("TCblockoffset"),
        py::arg("SparseAToX"), py::arg("num_nodes"), py::arg("num_edges"),
        py::arg("values") = py::none(), py::arg("bias") = py::none(), py::arg("relu") = false);
  // backward aliases of the reference (DTCSpMM.cpp:385-398): the same forward
  // functions, valid as a backward for symmetric A only
  m.def("backward_ptx_uint8_improved", &run_DTCSpMM, "alias of run_DTCSpMM", py::arg("X"),
        py::arg("RowWindowOffset"), py::arg("TCblocktileId"), py::arg("TCblockoffset"),
        py::arg("SparseAToX"), py::arg("num_nodes"), py::arg("num_edges"), py::arg("exeplan"),
        py::arg("values") = py::none());
  m.def("backward_ptx_uint8_improved_gcn", &DTCSpMM_gcn, "alias of DTCSpMM_gcn", py::arg("X"),
        py::arg("RowWindowOffset"), py::arg("TCblocktileId"), py::arg("TCblockoffset"),
        py::arg("SparseAToX"), py::arg("num_nodes"), py::arg("num_edges"),
        py::arg("values") = py::none(), py::arg("bias") = py::none(), py::arg("relu") = false);
  m.def("balance_backward_ptx_uint8_prefetch", &run_DTCSpMM_balance,
        "alias of run_DTCSpMM_balance", py::arg("X"), py::arg("TCblockRowid"),
        py::arg("TCblocktileId"), py::arg("TCblockoffset"), py::arg("SparseAToX"),
        py::arg("num_nodes"), py::arg("exeplan"), py::arg("values") = py::none());
  m.def("run_DTCSpMM_ex", &run_DTCSpMM_ex, "SpMM with a chosen B format / precision / schedule",
        py::arg("Bplanes"), py::arg("bformat"), py::arg("N"), py::arg("RowWindowOffset"),
        py::arg("TCblocktileId"), py::arg("TCblockoffset"), py::arg("SparseAToX"),
        py::arg("num_nodes"), py::arg("precision"), py::arg("mode") = 0, py::arg("grid") = 0,
        py::arg("values") = py::none(), py::arg("ntile") = 0, py::arg("block_h") = 16,
        py::arg("block_w") = 8);
  m.def("pack_b", &pack_b, "convert fp32 B into a storage form", py::arg("B"),
        py::arg("bformat"));
}
