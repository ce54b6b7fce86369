"""ctypes binding of the CUDA library (include/augur_b200.h).

The library is the only compute path: if libaugur_b200.so is missing or a
call fails, an AugurError is raised; there is no CPU fallback.
"""
import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libaugur_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "augur_b200.h")


class AugurError(RuntimeError):
    pass


_lib = None

i32, u32, u64, f64, f32 = C.c_int, C.c_uint32, C.c_uint64, C.c_double, C.c_float
# status codes of include/augur_b200.h
AB_OK, AB_ERR_ARG, AB_ERR_CUDA, AB_ERR_TIMEOUT, AB_ERR_NUMERIC, AB_ERR_STATE = range(6)
vp, sz = C.c_void_p, C.c_size_t


def header_symbols(path=HEADER):
    """Names of every function declared in the public header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ab_[a-z0-9_]+)\s*\(", text)))


def lib():
    """Loads libaugur_b200.so (building it first if the sources are newer is
    the job of augurv2_b200.build; this only loads)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AugurError(
                "CUDA library %s is missing: run `python -m augurv2_b200.build` "
                "(there is no CPU fallback)" % LIB_PATH)
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def last_error():
    return lib().ab_last_error().decode()


def check(rc, what=""):
    if rc != 0:
        raise AugurError("%s failed (status %d): %s" % (what, rc, last_error()))
    return rc


class LdaDesc(C.Structure):
    _fields_ = [("D", i32), ("K", i32), ("V", i32),
                ("doc_off", vp), ("w", vp), ("alpha", vp), ("beta", vp),
                ("z", vp), ("theta", vp), ("phiT", vp), ("cnt_dk", vp), ("cnt_kw", vp),
                ("scratch", vp), ("seed", u64)]


_dp, _ip = C.POINTER(C.c_double), C.POINTER(C.c_int)


class HlrCompC(C.Structure):
    _fields_ = [("kind", i32), ("P", i32), ("idx_off", i32), ("max_depth", i32), ("simlen", f64), ("eps", f64),
                ("mwg_var", f64)]


class LdaInit(C.Structure):
    """ab_lda_init: host arrays of an LDA model for ab_init_lda."""
    _fields_ = [("D", i32), ("K", i32), ("V", i32), ("doc_off", _ip), ("w", _ip), ("alpha", _dp), ("beta", _dp),
                ("theta", _dp), ("phi", _dp), ("z", _ip), ("seed", u64), ("iter0", u32)]


class HlrInit(C.Structure):
    """ab_hlr_init: host arrays of an HLR model and schedule for ab_init_hlr."""
    _fields_ = [("N", i32), ("D", i32), ("has_b", i32), ("vprior", i32), ("compat", i32), ("lam", f64),
                ("a0", f64), ("s0", f64), ("X", _dp), ("y", _ip), ("C", i32), ("pars", _dp), ("n_comps", i32),
                ("comps", C.POINTER(HlrCompC)), ("idx", _ip), ("n_idx", i32), ("seed", u64), ("iter0", u32)]


class GmmInit(C.Structure):
    """ab_gmm_init: host arrays of a Gaussian-mixture model for ab_init_gmm."""
    _fields_ = [("N", i32), ("d", i32), ("K", i32), ("shared_cov", i32), ("move", i32), ("compat", i32),
                ("Y", _dp), ("mu0", _dp), ("cov0", _dp), ("pis", _dp), ("covs", _dp), ("alpha", _dp), ("df", i32),
                ("scale0", _dp), ("prop_cov", _dp), ("mu", _dp), ("z", _ip), ("seed", u64), ("iter0", u32)]


_SIGS = {
    "ab_last_error": (C.c_char_p, []),
    "ab_version": (C.c_char_p, []),
    # LDA
    "ab_lda_phi_stride": (i32, [i32]),
    "ab_lda_count": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, vp]),
    "ab_lda_conj_theta": (i32, [i32, i32, vp, vp, vp, u64, u32, vp]),
    "ab_lda_phi_scratch_bytes": (sz, [i32, i32]),
    "ab_lda_conj_phi": (i32, [i32, i32, vp, vp, vp, i32, u64, u32, vp, vp]),
    "ab_lda_conj_phi_noalloc": (i32, [i32, i32, vp, vp, vp, i32, u64, u32, vp]),
    "ab_lda_disc_z": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, u64, u32, vp]),
    "ab_lda_scratch_bytes": (sz, [i32, i32]),
    "ab_lda_phi32_stride": (i32, [i32]),
    "ab_lda_disc_z_f32": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, u64, u32, vp]),
    "ab_lda_create": (i32, [C.POINTER(LdaDesc), C.POINTER(vp)]),
    "ab_lda_init_state": (i32, [vp, u32, vp]),
    "ab_lda_run": (i32, [vp, i32, i32, vp]),
    "ab_lda_destroy": (i32, [vp]),
    # HLR
    "ab_hlr_ll_grad": (i32, [vp, vp, vp, i32, i32, vp, vp, vp, vp]),
    "ab_hlr_chain_scratch_bytes": (sz, [i32, i32]),
    "ab_hlr_run_chains": (i32, [vp, vp, vp, i32, vp, vp, i32, vp, i32, u32, u64, vp, vp, vp]),
    # batched HLR, batched HMC, surrogate MLP
    "ab_hlrb_xt_elems": (sz, [i32, i32]),
    "ab_hlrb_transpose": (i32, [i32, i32, vp, i32, vp, vp]),
    "ab_hlrb_workspace_bytes": (sz, [i32, i32, i32]),
    "ab_hlrb_logp_grad": (i32, [vp, i32, vp, i32, vp, vp, i32, vp, vp, vp]),
    "ab_hlrb_workspace_bytes_cfg": (sz, [i32, i32, i32, vp]),
    "ab_hlrb_logp_grad_cfg": (i32, [vp, i32, vp, i32, vp, vp, i32, vp, vp, vp, vp]),
    "ab_nutsb_state_bytes": (sz, [i32, i32, i32]),
    "ab_nutsb_reset_history": (i32, [vp, i32, i32, i32, vp]),
    "ab_nutsb_init": (i32, [vp, i32, i32, i32, vp, vp, vp, u32, vp]),
    "ab_nutsb_thprop": (i32, [vp, i32, i32, i32, vp, vp, vp]),
    "ab_nutsb_advance": (i32, [vp, i32, i32, i32, i32, f64, u64, u32, vp, vp, vp]),
    "ab_nutsb_advance_variant": (i32, [vp, i32, i32, i32, i32, f64, u64, u32, i32, vp, vp, vp]),
    "ab_nutsb_info": (i32, [vp, i32, i32, i32, vp, vp]),
    "ab_hlrg_create": (i32, [i32, vp, vp, vp]),
    "ab_hlrg_bind": (i32, [vp, i32, vp, i32, vp, vp, i32]),
    "ab_hlrg_set_active": (i32, [vp, vp, vp]),
    "ab_hlrg_logp_grad": (i32, [vp, vp, vp]),
    "ab_hlrg_fused": (i32, [vp]),
    "ab_hlrg_destroy": (i32, [vp]),
    "ab_nutsg_create": (i32, [i32, vp, vp]),
    "ab_nutsg_set_active": (i32, [vp, vp, vp]),
    "ab_nutsg_advance": (i32, [vp, vp]),
    "ab_nutsg_min_draws": (i32, [vp, vp, vp]),
    "ab_nutsg_destroy": (i32, [vp]),
    "ab_hmcb_begin": (i32, [vp, vp]),
    "ab_hmcb_step": (i32, [vp, vp, vp]),
    "ab_hmcb_final": (i32, [vp, vp, vp, vp]),
    "ab_mlp_param_count": (sz, [i32, i32, i32, i32]),
    "ab_mlp_act_floats": (sz, [i32, i32, i32]),
    "ab_mlp_backward_scratch_floats": (sz, [i32, i32, i32]),
    "ab_mlp_forward": (i32, [vp, i32, vp, i32, vp, i32, vp, vp]),
    "ab_mlp_mse": (i32, [i32, i32, vp, i32, vp, i32, vp, vp, vp]),
    "ab_mlp_backward": (i32, [vp, i32, vp, i32, vp, vp, vp, vp, vp]),
    "ab_mlp_adam": (i32, [vp, vp, vp, vp, i32, f32, f32, f32, f32, vp]),
    "ab_mlp_sync_bf16": (i32, [vp, vp]),
    "ab_sur_pre": (i32, [i32, i32, vp, vp, vp, vp, vp]),
    "ab_sur_predict": (i32, [vp, i32, vp, i32, vp, vp, vp, vp, vp, vp, i32, vp]),
    "ab_sur_post": (i32, [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp]),
    # tensor-core GEMM core
    "ab_tc_gemm_bf16": (i32, [i32, i32, i32, vp, i32, vp, i32, vp, i32, i32, vp, vp]),
    "ab_tc_wait_probe": (i32, [C.c_longlong, vp, vp, vp]),
    # scalar conjugate updates
    "ab_conj_scalar": (i32, [i32, i32, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, u64, u32, vp]),
    # GMM
    "ab_gmm_table_doubles": (sz, [i32, i32]),
    "ab_gmm_prep": (i32, [i32, i32, vp, vp, vp, vp]),
    "ab_gmm_disc_z": (i32, [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, u64, u32, u32, vp]),
    "ab_gmm_z_scratch_bytes": (sz, [i32, i32, i32]),
    "ab_gmm_z_queue_offset": (sz, [i32, i32]),
    "ab_gmm_disc_z_screened": (i32, [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, u64, u32, u32, vp, vp]),
    "ab_gmm_stats_scratch_bytes": (sz, [i32, i32]),
    "ab_gmm_stats": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp]),
    "ab_gmm_conj_pis": (i32, [i32, vp, vp, vp, u64, u32, u32, vp]),
    "ab_gmm_conj_mu": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, vp, u64, u32, u32, vp]),
    "ab_gmm_conj_cov": (i32, [i32, i32, i32, vp, vp, vp, vp, u64, u32, u32, vp]),
    "ab_gmm_bartlett": (i32, [i32, i32, i32, vp, vp, u64, u32, u32, vp]),
    "ab_gmm_conj_cov_chi": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, u64, u32, u32, vp]),
    "ab_gmm_eslice": (i32, [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32, vp, u64, u32, u32, vp, vp]),
    "ab_gmm_mwg": (i32, [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32, i32, i32, vp, u64, u32, u32, vp, vp]),
    # whole-model log densities, predictive log-likelihoods, dethlr's bias
    "ab_ll_scratch_bytes": (sz, []),
    "ab_lda_ll_mod": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "ab_lda_pred_ll": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp]),
    "ab_gmm_ll_mod": (i32, [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp,
                            vp]),
    "ab_gmm_pred_ll": (i32, [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp]),
    "ab_hlr_det": (i32, [vp, i32, vp, vp, vp]),
    # model handles
    "ab_init_lda": (i32, [C.POINTER(LdaInit), C.POINTER(vp)]),
    "ab_init_hlr": (i32, [C.POINTER(HlrInit), C.POINTER(vp)]),
    "ab_init_gmm": (i32, [C.POINTER(GmmInit), C.POINTER(vp)]),
    "ab_model_kind": (i32, [vp]),
    "ab_model_last_error": (C.c_char_p, [vp]),
    "ab_step": (i32, [vp, i32, vp]),
    "ab_iteration": (u32, [vp]),
    "ab_state_bytes": (sz, [vp]),
    "ab_get_state": (i32, [vp, vp, sz, vp]),
    "ab_set_state": (i32, [vp, vp, sz, vp]),
    "ab_checkpoint_bytes": (sz, [vp]),
    "ab_checkpoint": (i32, [vp, vp, sz, vp]),
    "ab_restore": (i32, [vp, vp, sz, vp]),
    "ab_curr_ll_count": (i32, [vp]),
    "ab_curr_ll": (i32, [vp, _dp, i32, vp]),
    "ab_destroy": (i32, [vp]),
}


def _declare(L):
    for name, (res, args) in _SIGS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def stream_ptr(stream=None):
    """cudaStream_t of a torch stream (current stream by default)."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    return None if t is None else C.c_void_p(t.data_ptr())
