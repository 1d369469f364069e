"""ctypes mirror of include/intspmv.h: the reference's structs, field for
field (edoardoCB/int_spmv intSpmv_main.c:183,306,400,429,615,771,1114), and
the prototypes of every exported function."""
from __future__ import annotations

import ctypes as C

UIN = C.c_uint
FPT = C.c_double
P_UIN = C.POINTER(UIN)
P_FPT = C.POINTER(FPT)
P_P_UIN = C.POINTER(P_UIN)
VP = C.c_void_p


class StrMatCSR(C.Structure):  # intSpmv_main.c:183
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("rmin", UIN), ("rave", FPT), ("rmax", UIN), ("rsd", FPT),
                ("bw", UIN), ("val", P_FPT), ("row", P_UIN), ("rowStart", P_UIN), ("rowEnd", P_UIN),
                ("col", P_UIN), ("rl", P_UIN)]


class StrFormatData(C.Structure):  # intSpmv_main.c:306
    _fields_ = [("name", C.c_char * 24), ("mfp", C.c_double), ("beta", C.c_double), ("ct", C.c_double)]


class StrErr(C.Structure):  # intSpmv_main.c:400
    _fields_ = [("aErr", C.c_double), ("rErr", C.c_double), ("pos", UIN)]


class StrRes(C.Structure):  # intSpmv_main.c:429
    _fields_ = [("name", C.c_char * 25), ("et", C.c_double), ("ot", C.c_double), ("flops", C.c_double),
                ("sErr", StrErr)]


class StrMatAXC(C.Structure):  # intSpmv_main.c:615
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("lenAX", UIN), ("lenBRP", UIN), ("ax", P_FPT), ("brp", P_UIN)]


class StrMatK1(C.Structure):  # intSpmv_main.c:771
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("chunkNum", UIN), ("lenVC", UIN), ("permi", P_UIN), ("nmc", P_UIN),
                ("chp", P_UIN), ("val", P_FPT), ("col", P_UIN)]


class StrMatAXT(C.Structure):  # intSpmv_main.c:1114
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("mode", C.c_char * 8), ("tileHW", UIN), ("tileH", UIN),
                ("logTH", UIN), ("tileN", UIN), ("lenAX", UIN), ("lenSEC", UIN), ("lenCON", UIN), ("log", UIN),
                ("ax", P_FPT), ("sec", P_UIN), ("con", P_UIN)]


class PlanOpts(C.Structure):
    _fields_ = [("val_kind", C.c_int), ("col_kind", C.c_int), ("kernel", C.c_int), ("ctas_per_sm", C.c_int),
                ("units_per_warp", C.c_int), ("lo_tol", C.c_double), ("variant", C.c_int), ("rhs_block", C.c_int),
                ("spmm_kernel", C.c_int)]


class PlanInfo(C.Structure):
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("slots", C.c_uint64), ("device_bytes", C.c_uint64),
                ("alg_bytes", C.c_double), ("format", C.c_int), ("val_kind", C.c_int), ("col_kind", C.c_int),
                ("kernel", C.c_int), ("tile_h", UIN), ("bs", UIN), ("name", C.c_char * 32)]


class PlanLayout(C.Structure):
    _fields_ = [("slots", C.c_uint64), ("slots_pad", C.c_uint64), ("seg_slots", C.c_uint64), ("nseg", C.c_uint64),
                ("nrowmap", C.c_uint64), ("nempty", C.c_uint64), ("val_bytes", UIN), ("spl", UIN),
                ("nwin", C.c_uint64)]


P_CSR = C.POINTER(StrMatCSR)
P_FD = C.POINTER(StrFormatData)
P_AXC = C.POINTER(StrMatAXC)
P_K1 = C.POINTER(StrMatK1)
P_AXT = C.POINTER(StrMatAXT)
P_OPTS = C.POINTER(PlanOpts)
P_PLAN = C.POINTER(VP)

# name: (restype, argtypes).  Every `extern "C"` function of include/intspmv.h.
PROTOTYPES: dict[str, tuple] = {
    # format conversion on the GPU
    "ispmv_dev_build_axt": (C.c_int, [UIN, UIN, UIN, C.c_char_p, UIN, UIN, VP, VP, VP, VP,
                                      C.POINTER(StrMatAXT), C.POINTER(StrFormatData), VP]),
    "ispmv_dev_axt_free": (C.c_int, [C.POINTER(StrMatAXT)]),
    "ispmv_dev_axt_export": (C.c_int, [C.POINTER(StrMatAXT), VP, VP, VP, VP]),
    "ispmv_dev_build_k1": (C.c_int, [UIN, UIN, VP, VP, VP, C.POINTER(StrMatK1), C.POINTER(StrFormatData), VP]),
    "ispmv_dev_k1_free": (C.c_int, [C.POINTER(StrMatK1)]),
    "ispmv_dev_k1_export": (C.c_int, [C.POINTER(StrMatK1), VP, VP, VP, VP, VP, VP]),
    # self-test of the bounded device wait
    "ispmv_selftest_bounded_wait": (C.c_int, [C.POINTER(C.c_double), C.c_void_p]),
    # host: statistics, files, builders
    "ispmv_csr_stats": (C.c_int, [P_CSR]),
    "printMatrixStats": (None, [C.c_char_p, P_CSR]),
    "ispmv_matrix_read": (C.c_int, [C.c_char_p, P_CSR]),
    "matrixReading": (StrMatCSR, [C.c_char_p]),
    "ispmv_matrix_write": (C.c_int, [C.c_char_p, P_CSR]),
    "ispmv_csr_free": (None, [P_CSR]),
    "ispmv_build_csr": (C.c_int, [P_CSR, P_FD]),
    "getFormatDataCSR": (StrFormatData, [P_CSR]),
    "ispmv_build_axc": (C.c_int, [UIN, P_CSR, P_FPT, P_AXC, P_FD]),
    "getFormatDataAXC": (StrFormatData, [UIN, StrMatCSR, P_FPT, P_AXC]),
    "ispmv_build_k1": (C.c_int, [UIN, P_CSR, P_FPT, P_K1, P_FD]),
    "getFormatDataK1": (StrFormatData, [UIN, StrMatCSR, P_FPT, P_K1]),
    "ispmv_build_axt": (C.c_int, [UIN, UIN, UIN, UIN, C.c_char_p, P_CSR, P_FPT, P_AXT, P_FD]),
    "getFormatDataAXT": (StrFormatData, [UIN, UIN, UIN, UIN, C.c_char_p, StrMatCSR, P_FPT, P_AXT]),
    "ispmv_build_axc_cols": (C.c_int, [UIN, P_CSR, P_AXC, P_P_UIN]),
    "ispmv_build_axt_cols": (C.c_int, [UIN, P_CSR, P_AXT, P_P_UIN]),
    "ispmv_csr_blockdiag": (C.c_int, [UIN, P_CSR, P_CSR, P_UIN]),
    "ispmv_gen_banded": (C.c_int, [UIN, C.c_uint64, UIN, UIN, UIN, P_CSR]),
    "ispmv_free_axc": (None, [P_AXC]),
    "ispmv_free_k1": (None, [P_K1]),
    "ispmv_free_axt": (None, [P_AXT]),
    "getErrors": (None, [UIN, P_FPT, P_FPT, C.POINTER(StrErr)]),
    "initVec": (None, [UIN, P_FPT]),
    "fill_array": (None, [UIN, UIN, C.c_double, P_FPT]),
    # the reference's per-kernel harness (test_*), runs per call
    "ispmv_set_num_ite": (None, [UIN]),
    "ispmv_get_num_ite": (UIN, []),
    "test_cf_CSR": (StrRes, [StrMatCSR, P_FPT, P_FPT]),
    "test_int_AXC": (StrRes, [UIN, StrMatAXC, P_FPT]),
    "test_int_k1": (StrRes, [UIN, StrMatK1, P_FPT, P_FPT]),
    "test_int_k1p": (StrRes, [UIN, StrMatK1, P_FPT, P_FPT]),
    "test_int_axt_noc_h1": (StrRes, [UIN, StrMatAXT, P_FPT]),
    "test_int_axt_noc": (StrRes, [UIN, StrMatAXT, P_FPT]),
    "test_int_axt_com_h1": (StrRes, [UIN, UIN, StrMatAXT, P_FPT]),
    # device kernels on device pointers
    "ispmv_dev_cf_csr": (C.c_int, [UIN, VP, VP, VP, VP, VP, VP]),
    "ispmv_dev_int_axc": (C.c_int, [UIN, VP, VP, VP, VP]),
    "ispmv_dev_int_k1": (C.c_int, [UIN, VP, VP, VP, VP, VP, VP, VP]),
    "ispmv_dev_order_k1": (C.c_int, [UIN, VP, VP, VP, VP]),
    "ispmv_dev_int_k1p": (C.c_int, [C.c_ubyte, UIN, VP, VP, VP, VP, VP, VP, VP, VP]),
    "ispmv_dev_int_axt_noc_h1": (C.c_int, [UIN, VP, VP, VP, VP]),
    "ispmv_dev_int_axt_noc": (C.c_int, [UIN, UIN, VP, VP, VP, VP]),
    "ispmv_dev_int_axt_com_h1": (C.c_int, [UIN, UIN, UIN, UIN, UIN, UIN, UIN, VP, VP, VP, VP]),
    "ispmv_dev_k1_spmv_noalloc": (C.c_int, [UIN, UIN, VP, VP, VP, VP, VP, VP, VP, VP]),
    # the reference's kernels by name, on host pointers
    "cf_CSR": (None, [StrMatCSR, P_FPT, P_FPT]),
    "int_axc": (None, [UIN, UIN, P_FPT, P_UIN, P_FPT]),
    "int_k1": (None, [UIN, UIN, P_FPT, P_UIN, P_UIN, P_UIN, P_FPT, P_FPT]),
    "orderArrayK1": (None, [UIN, UIN, P_UIN, P_FPT, P_FPT]),
    "int_k1p": (None, [UIN, C.c_ubyte, UIN, P_FPT, P_UIN, P_UIN, P_UIN, P_UIN, P_FPT, P_FPT]),
    "int_axt_noc_h1": (None, [UIN, UIN, P_FPT, P_UIN, P_FPT]),
    "int_axt_noc": (None, [UIN, UIN, UIN, P_FPT, P_UIN, P_FPT]),
    "int_axt_com_h1": (None, [UIN, UIN, UIN, UIN, UIN, UIN, UIN, UIN, P_FPT, P_UIN, P_FPT]),
    # plans
    "ispmv_plan_opts_default": (None, [P_OPTS]),
    "ispmv_plan_csr": (C.c_int, [P_CSR, P_OPTS, P_PLAN]),
    "ispmv_plan_axc": (C.c_int, [P_CSR, P_AXC, P_UIN, P_OPTS, P_PLAN]),
    "ispmv_plan_k1": (C.c_int, [P_CSR, P_K1, C.c_int, P_OPTS, P_PLAN]),
    "ispmv_plan_axt": (C.c_int, [P_CSR, P_AXT, P_UIN, P_OPTS, P_PLAN]),
    "ispmv_plan_dev_csr": (C.c_int, [UIN, UIN, VP, VP, VP, P_OPTS, P_PLAN, VP]),
    "ispmv_plan_get_layout": (C.c_int, [VP, C.POINTER(PlanLayout)]),
    "ispmv_plan_export_stream": (C.c_int, [VP, VP, VP, VP, VP, VP, VP, VP]),
    "ispmv_plan_export_windows": (C.c_int, [VP, VP, VP, VP]),
    "ispmv_plan_destroy": (C.c_int, [VP]),
    "ispmv_plan_spmv": (C.c_int, [VP, VP, VP, C.c_int, VP]),
    "ispmv_plan_spmv_graph": (C.c_int, [VP, VP, VP, C.c_int, VP]),
    "ispmv_plan_spmm": (C.c_int, [VP, UIN, VP, VP, VP]),
    "ispmv_plan_spmv_host": (C.c_int, [VP, VP, VP, VP]),
    "ispmv_plan_get_info": (C.c_int, [VP, C.POINTER(PlanInfo)]),
    "ispmv_plan_status": (C.c_int, [VP]),
    "ispmv_plan_time_kernels": (C.c_int, [VP, C.c_int]),
    "ispmv_plan_kernel_ms": (C.c_int, [VP, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "ispmv_plan_time_main": (C.c_int, [VP, VP, VP, C.c_int, VP, C.POINTER(C.c_double)]),
    "ispmv_plan_kernel_name": (C.c_char_p, [VP]),
    # library facts
    "ispmv_version": (C.c_char_p, []),
    "ispmv_status_string": (C.c_char_p, [C.c_int]),
    "ispmv_last_error": (C.c_char_p, []),
    "ispmv_launch_count": (C.c_ulonglong, []),
}

# status codes (include/intspmv.h)
OK, ERR_ARG, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_OVERFLOW = range(7)
VAL_F64, VAL_F32, VAL_F32_LO16 = 0, 1, 2
COL_U32, COL_D16 = 0, 1
KERNEL_AUTO, KERNEL_LDG, KERNEL_TMA, KERNEL_ROWS, KERNEL_WIDE = 0, 1, 2, 3, 4
VARIANT_QUEUE = 16
