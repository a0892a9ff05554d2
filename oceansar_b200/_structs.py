"""ctypes mirrors of the descriptor structs in ``include/oceansar_b200.h`` (same field order)."""
import ctypes

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
F64 = ctypes.c_double
F32 = ctypes.c_float


class PulseDesc(ctypes.Structure):
    _fields_ = [("nx", I32), ("ny", I32), ("npol", I32), ("pol", I32), ("nch", I32),
                ("dx_d", P), ("dy_d", P), ("dz_d", P), ("diffx_d", P), ("diffy_d", P),
                ("diffxx_d", P), ("diffyy_d", P), ("diffxy_d", P), ("hmtf_d", P),
                ("y_d", P),
                ("sr_col_d", P), ("sin_inc_d", P), ("cos_inc_d", P), ("tan_inc_d", P), ("inc_d", P),
                ("c_b_d", P),
                ("inc_angle", F64), ("sr0", F64), ("gr0", F64), ("k0", F64), ("f0", F64),
                ("az_now", F64), ("min_sr", F64), ("binsize", F64), ("t_step", F64),
                ("az_step", I32), ("az_steps", I32), ("tind", I64),
                ("ant_l_tx", F64), ("ant_l_rx", F64),
                ("b_ati", ctypes.POINTER(F64)), ("b_xti", ctypes.POINTER(F64)),
                ("do_kodis", I32), ("do_bragg", I32), ("refresh", I32), ("use_hmtf", I32),
                ("kodis_R_re", F64), ("kodis_R_im", F64),
                ("facet_dx", F32), ("facet_dy", F32),
                ("bragg_d", F64), ("wind_dir", F64), ("wind_U", F64),
                ("spread", I32),
                ("spread_ck_p", F64), ("spread_ck_m", F64), ("spread_a0", F64), ("spread_ap", F64),
                ("spread_am", F64),
                ("spec_k_d", P), ("spec_s_d", P), ("spec_n", I32),
                ("sqrt_eps_re", F64), ("sqrt_eps_im", F64),
                ("scat_d", P), ("s_m_d", P), ("s_p_d", P), ("n_m", I64), ("n_p", I64),
                ("ind0_m_d", P), ("ind0_p_d", P),
                ("sinc_d", P), ("raw_d", P), ("nbins", I32),
                ("nrcs_spec_d", P), ("nrcs_bragg_d", P), ("rowtab_d", P),
                ("lut_d", P), ("lut_naz", I32), ("lut_ndy", I32), ("lut_ndx", I32),
                ("lut_az0", F64), ("lut_daz", F64), ("lut_dy0", F64), ("lut_ddy", F64),
                ("lut_dx0", F64), ("lut_ddx", F64),
                ("spec_mode", I32), ("x_d", P), ("ka_dx", F64), ("ka_dy", F64), ("ka_K_re", F64), ("ka_K_im", F64),
                ("s_m32_d", P), ("s_p32_d", P), ("sca", I32), ("field_nx", I32), ("roll", I32),
                ("sr_bin_offset", F64), ("cap_t", F64), ("nrcs_row", I32), ("nrcs_rows", I32),
                ("az_f32", I32), ("skim", I32), ("skim_ny_integ", I32), ("skim_az2", I32), ("skim_rcm", I32),
                ("raw_lo_d", P), ("pt_mode", I32), ("pt_x", I32), ("pt_y", I32), ("pt_amp", F64),
                ("lut_block", ctypes.c_int64)]


class RcsDesc(ctypes.Structure):
    _fields_ = [("nx", I32), ("ny", I32),
                ("az_d", P), ("az_row_stride", I64), ("az_col_stride", I64),
                ("inc_d", P), ("inc_row_stride", I64), ("inc_col_stride", I64),
                ("diffx_d", P), ("diffy_d", P),
                ("k0", F64), ("d", F64), ("dx", F64), ("dy", F64), ("wind_dir", F64), ("wind_U", F64),
                ("pol", I32), ("spread", I32),
                ("spread_ck_p", F64), ("spread_ck_m", F64), ("spread_a0", F64), ("spread_ap", F64),
                ("spread_am", F64),
                ("spec_k_d", P), ("spec_s_d", P), ("spec_n", I32),
                ("sqrt_eps_re", F64), ("sqrt_eps_im", F64),
                ("out_hh_d", P), ("out_vv_d", P)]


class KodisDesc(ctypes.Structure):
    _fields_ = [("nx", I32), ("ny", I32),
                ("az_d", P), ("az_row_stride", I64), ("az_col_stride", I64),
                ("sin_inc_d", P), ("cos_inc_d", P), ("tan_inc_d", P), ("sr_d", P),
                ("diffx_d", P), ("diffy_d", P), ("diffxx_d", P), ("diffyy_d", P), ("diffxy_d", P),
                ("k0", F64), ("R_re", F64), ("R_im", F64), ("dx", F64), ("dy", F64),
                ("out_d", P)]


class SceneDesc(ctypes.Structure):
    """``ocs_scene_desc``: one scene of the scene batch."""
    _fields_ = [("surface", ctypes.c_void_p), ("pulse", ctypes.c_void_p), ("tile_rows", ctypes.c_int32),
                ("t_d", ctypes.c_void_p), ("add_d", ctypes.c_void_p), ("swell_rot_d", ctypes.c_void_p),
                ("az_now_d", ctypes.c_void_p), ("flags_d", ctypes.c_void_p), ("tmod_d", ctypes.c_void_p),
                ("choppy", ctypes.c_void_p)]


class KaDesc(ctypes.Structure):
    """``ocs_ka_desc``: Kirchhoff-approximation field."""
    _fields_ = [("nx", I32), ("ny", I32), ("x_d", P), ("y_d", P),
                ("theta_d", P), ("theta_row_stride", I64), ("theta_col_stride", I64),
                ("phi_d", P), ("phi_row_stride", I64), ("phi_col_stride", I64),
                ("dz_d", P), ("diffx_d", P), ("diffy_d", P), ("diffxx_d", P), ("diffyy_d", P), ("diffxy_d", P),
                ("k0", F64), ("dx", F64), ("dy", F64), ("K_re", F64), ("K_im", F64),
                ("mode", I32), ("pol_i", I32), ("pol_s", I32), ("out_d", P)]
