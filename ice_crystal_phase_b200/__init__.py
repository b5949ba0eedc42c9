"""B200-native phase-function generation: Python mirror of the reference's stage interfaces.

The compute path is the CUDA shared library ``libicp_b200.so`` (C ABI, include/icp_b200.h)
built for sm_100a.  This module only marshals arguments: there is no CPU fallback, and
importing it raises if the library is missing.

Mirrored reference interfaces (Somatic-Cell/ice-crystal-phase):
  make_phase_grid / PhaseGrid      hex_phase/include/ice_crystal/phase_table.hpp:118-127
  rotation_from_quaternion         hex_phase/src/phase_table.cpp:11-21
  parse_orientation_plan           hex_phase/src/orientation_plan.cpp:69-120
  PhaseMassAccumulatorCuda         hex_phase/include/ice_crystal/phase_cuda.hpp:17-35
    (.add fused with HexPrismTracer.trace, hex_trace/include/ice_crystal/hex_trace_cuda.hpp:18-41)
  PhaseCdf.build                   include/rainbow/phase_cdf.hpp:50-96
  generate_hex_record              hex_phase/apps/generate_hex_phase.cpp:79-154 (CUDA branch)
  evaluate_water_optics            include/rainbow/water_refractive_index.hpp:22-33
  RaindropShape.make               include/rainbow/raindrop_shape.hpp:22-67
  compute_projected_area           include/rainbow/projected_area.hpp:31-35
  drop_frame                       apps/generate_phase.cpp:209-217, 242-245
  PhaseMassAccumulatorCuda.add_drop  RaindropTracer::trace_unpolarized + patch stages, replaced by
                                   direct binning (include/rainbow/raindrop_tracer.hpp:32-36)
  generate_drop_record             apps/generate_phase.cpp:395-453 (rainbow_generate's record path)
  patch_build                      PatchAccel::build's kernels, device/patch_build.cu:13-77
  query_directions                 QueryDirectionGrid::directions, include/rainbow/query_direction_grid.hpp:14-58
  patch_query                      PatchQuery::query_grid (OptiX all-hit query), src/patch_query.cpp
  patch_optics                     PatchOptics::evaluate_device / evaluate_wave_device's kernels
                                   evaluate_patch_optics / evaluate_focal_optics, device/patch_optics.cu:7-24
  stage_density / stage_record     density() + phase_check_density (device/phase_cdf.cu:40-108) and
                                   the CDF input gate (src/phase_cdf.cpp:325-328) before PhaseCdf::build
  rainbow_table_sigma              include/rainbow/rainbow_diffraction.hpp:16-28
  diffraction_config               src/patch_optics.cpp:79-95 (the diffraction part of evaluate_wave_device)
  rainbow_diffraction              PatchOptics::run_diffraction + its statistics, src/patch_optics.cpp:217-231,
                                   334-348 (kernels device/patch_optics.cu:26-40)
"""
from __future__ import annotations

import ctypes as C
import hashlib
import math
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libicp_b200.so"

ICP_OK, ICP_ERR_INVALID_ARGUMENT, ICP_ERR_AUDIT, ICP_ERR_CAPACITY, ICP_ERR_DEVICE, ICP_ERR_TIMEOUT, ICP_ERR_STATE = range(7)
ICP_FP32, ICP_FP64 = 0, 1
STATUS_NAMES = ["exhausted", "tail_tolerance_reached", "interaction_limit", "ambiguous_boundary", "invalid_input",
                "numerical_failure", "output_overflow", "replay_mismatch"]


class IcpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class InvalidArgument(IcpError, ValueError):
    pass


class AuditError(IcpError):
    pass


class CapacityError(IcpError):
    pass


_ERRORS = {ICP_ERR_INVALID_ARGUMENT: InvalidArgument, ICP_ERR_AUDIT: AuditError, ICP_ERR_CAPACITY: CapacityError}


# ---------------------------------------------------------------- ABI structures
class Grid(C.Structure):
    _fields_ = [("nt", C.c_uint32), ("np", C.c_uint32), ("ki", C.c_double * 3), ("e0", C.c_double * 3),
                ("e1", C.c_double * 3)]


class TraceStats(C.Structure):
    _fields_ = [("escaped", C.c_double), ("unresolved", C.c_double), ("point_axial", C.c_double),
                ("forward_pole", C.c_double), ("backward_pole", C.c_double), ("max_ray_balance", C.c_double),
                ("max_interface_balance", C.c_double), ("rays", C.c_uint64), ("outputs", C.c_uint64),
                ("status_counts", C.c_uint64 * 8), ("rejected_rays", C.c_uint64), ("snapped", C.c_uint64),
                ("near_edge", C.c_uint64), ("fallback_adds", C.c_uint64), ("max_batch_outputs", C.c_uint64),
                ("invalid", C.c_uint64), ("encounters", C.c_uint64), ("missed", C.c_uint64),
                ("gauge_evals", C.c_uint64)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "status_counts"}
        d["status_counts"] = {STATUS_NAMES[i]: int(self.status_counts[i]) for i in range(8)}
        return d


class Tuning(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("hash_slots", C.c_uint32),
                ("reserved", C.c_uint32)]


class HexNode(C.Structure):
    _fields_ = [("circumradius_mm", C.c_double), ("length_mm", C.c_double), ("rotation", C.c_double * 9),
                ("exterior_index", C.c_double), ("interior_index", C.c_double), ("tail_tolerance", C.c_double),
                ("balance_tolerance", C.c_double), ("area_weight", C.c_double), ("seed", C.c_uint64),
                ("total_samples", C.c_uint64), ("first_sample", C.c_uint64), ("sample_count", C.c_uint64),
                ("max_internal_hits", C.c_uint32), ("batch_size", C.c_uint32), ("precision", C.c_uint32),
                ("reserved", C.c_uint32)]


class CdfPolicy(C.Structure):
    _fields_ = [("max_l1_error", C.c_double), ("max_lost_mass", C.c_double), ("max_coarsening_tv", C.c_double)]


class CdfReport(C.Structure):
    _fields_ = [("g_source", C.c_double), ("g_stored", C.c_double), ("coarsening_tv", C.c_double),
                ("cdf_mass", C.c_double), ("l1_error", C.c_double), ("lost_mass", C.c_double),
                ("maximum_cell_error", C.c_double), ("aggregation_relative_error", C.c_double),
                ("fine_mass", C.c_double), ("fine_axial", C.c_double), ("lost_cells", C.c_uint64),
                ("malformed", C.c_uint64), ("status", C.c_uint32), ("reserved", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class HexRecordArgs(C.Structure):
    _fields_ = [("circumradius_mm", C.c_double), ("length_mm", C.c_double), ("ki", C.c_double * 3),
                ("exterior_index", C.c_double), ("interior_index", C.c_double), ("tail_tolerance", C.c_double),
                ("balance_tolerance", C.c_double), ("nt", C.c_uint32), ("np", C.c_uint32), ("ct", C.c_uint32),
                ("cp", C.c_uint32), ("max_internal_hits", C.c_uint32), ("batch_size", C.c_uint32),
                ("max_output_records", C.c_uint64), ("precision", C.c_uint32), ("reserved", C.c_uint32),
                ("policy", CdfPolicy), ("tuning", Tuning)]


class Orientation(C.Structure):
    _fields_ = [("quaternion", C.c_double * 4), ("weight", C.c_double), ("samples", C.c_uint64), ("seed", C.c_uint64)]


class RecordReport(C.Structure):
    _fields_ = [("trace", TraceStats), ("expected_area_mm2", C.c_double), ("escaped_area_mm2", C.c_double),
                ("unresolved_area_mm2", C.c_double), ("histogram_mass_mm2", C.c_double),
                ("histogram_axial_mm2", C.c_double), ("point_mass_mm2", C.c_double), ("point_axial_mm2", C.c_double),
                ("forward_mass_mm2", C.c_double), ("backward_mass_mm2", C.c_double),
                ("histogram_relative_error", C.c_double), ("cdf", CdfReport), ("seconds_trace", C.c_double),
                ("seconds_cdf", C.c_double)]


class DropRecordArgs(C.Structure):
    _fields_ = [("radius_mm", C.c_double), ("coefficients", C.c_double * 8), ("inclination_deg", C.c_double),
                ("exterior_index", C.c_double), ("interior_index", C.c_double), ("wavelength_nm", C.c_double),
                ("tail_tolerance", C.c_double), ("balance_tolerance", C.c_double), ("nt", C.c_uint32),
                ("np", C.c_uint32), ("ct", C.c_uint32), ("cp", C.c_uint32), ("max_internal_hits", C.c_uint32),
                ("precision", C.c_uint32), ("rays", C.c_uint64), ("seed", C.c_uint64), ("diffraction", C.c_uint32),
                ("reserved", C.c_uint32), ("policy", CdfPolicy), ("tuning", Tuning)]


class DropReport(C.Structure):
    _fields_ = [("trace", TraceStats), ("projected_area_mm2", C.c_double), ("sampled_area_mm2", C.c_double),
                ("incident_area_mm2", C.c_double), ("escaped_area_mm2", C.c_double),
                ("unresolved_area_mm2", C.c_double), ("diffraction_area_mm2", C.c_double),
                ("forward_mass_mm2", C.c_double), ("backward_mass_mm2", C.c_double),
                ("histogram_mass_mm2", C.c_double), ("point_axial_mm2", C.c_double),
                ("histogram_relative_error", C.c_double), ("ki", C.c_double * 3), ("e0", C.c_double * 3),
                ("e1", C.c_double * 3), ("cdf", CdfReport), ("seconds_trace", C.c_double),
                ("seconds_cdf", C.c_double)]


class DropItem(C.Structure):
    _fields_ = [("radius_mm", C.c_double), ("coefficients", C.c_double * 8), ("inclination_deg", C.c_double),
                ("interior_index", C.c_double), ("wavelength_nm", C.c_double), ("rays", C.c_uint64),
                ("seed", C.c_uint64), ("diffraction", C.c_uint32), ("reserved", C.c_uint32)]


class BatchSettings(C.Structure):
    _fields_ = [("nt", C.c_uint32), ("np", C.c_uint32), ("ct", C.c_uint32), ("cp", C.c_uint32),
                ("max_internal_hits", C.c_uint32), ("precision", C.c_uint32), ("exterior_index", C.c_double),
                ("tail_tolerance", C.c_double), ("balance_tolerance", C.c_double), ("policy", CdfPolicy),
                ("block_threads", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("chunk_rays", C.c_uint32),
                ("use_graph", C.c_uint32)]


class IceState(C.Structure):
    _fields_ = [("wavelength_nm", C.c_double), ("n", C.c_double), ("kappa", C.c_double), ("lower_nm", C.c_double),
                ("upper_nm", C.c_double), ("log_wavelength_fraction", C.c_double)]


class AtlasRay(C.Structure):
    _fields_ = [("face", C.c_uint32), ("reserved", C.c_uint32), ("x", C.c_double), ("y", C.c_double),
                ("z", C.c_double), ("weight_mm2", C.c_double)]


class AtlasIncident(C.Structure):
    _fields_ = [("theta", C.c_double), ("phi", C.c_double), ("ki", C.c_double * 3), ("e0", C.c_double * 3),
                ("e1", C.c_double * 3), ("rule_ki", C.c_double * 3)]


class AtlasSettings(C.Structure):
    _fields_ = [("circumradius_mm", C.c_double), ("length_mm", C.c_double), ("interior_index", C.c_double),
                ("exterior_index", C.c_double), ("theta_intervals", C.c_uint32), ("phi_intervals", C.c_uint32),
                ("nt", C.c_uint32), ("np", C.c_uint32), ("subdivisions", C.c_uint32),
                ("max_internal_hits", C.c_uint32), ("tail_tolerance", C.c_double),
                ("max_unresolved_fraction", C.c_double), ("max_balance_error", C.c_double)]


class AtlasNodeReport(C.Structure):
    _fields_ = [("projected_area_mm2", C.c_double), ("escaped_mm2", C.c_double), ("unresolved_mm2", C.c_double),
                ("histogram_mass_mm2", C.c_double), ("histogram_relative_error", C.c_double),
                ("max_balance_error", C.c_double), ("max_interface_balance_error", C.c_double),
                ("rays", C.c_uint64), ("outputs", C.c_uint64), ("invalid_bins", C.c_uint64),
                ("status", C.c_uint64 * 8), ("first_rejected", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: (list(getattr(self, k)) if k == "status" else getattr(self, k)) for k, _ in self._fields_}


class DiffractionConfig(C.Structure):
    _fields_ = [("primary_sigma_rad", C.c_double), ("support_sigma", C.c_double),
                ("transition_contrast", C.c_double), ("inner_blend_sigma", C.c_double)]


class DiffractionStats(C.Structure):
    _fields_ = [(k, C.c_uint32) for k in ("primary_transitions", "secondary_transitions", "unknown_transitions",
                                          "filtered_directions", "unavailable_directions",
                                          "underresolved_directions")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


# One focal-stage query direction (icp_focal_sample = rainbow::FocalOpticalResult, 144 bytes) and
# one diffraction result (icp_diffraction_result = rainbow::DiffractionResult, 40 bytes).
FOCAL_DTYPE = np.dtype([("field", "<f8", 4), ("intensity_s", "<f8"), ("intensity_p", "<f8"),
                        ("family_incoherent", "<f8", 4), ("family_hits", "<u4", 4), ("corrected_hits", "<u4"),
                        ("extra_quarter_turn_hits", "<u4"), ("flags", "<u4"), ("first_problem_patch_id", "<u4"),
                        ("field_second", "<f8", 4)])
DIFFRACTION_DTYPE = np.dtype([("intensity_s", "<f8"), ("intensity_p", "<f8"), ("sigma_rad", "<f8"),
                              ("blend", "<f8"), ("flags", "<u4"), ("transition_kind", "<u4")])
TRANSITION_PRIMARY, TRANSITION_SECONDARY, TRANSITION_UNKNOWN = 1, 2, 4
DIFFRACTION_FILTERED, DIFFRACTION_UNDERRESOLVED, DIFFRACTION_INPUT_UNAVAILABLE = 1, 2, 4
DIFFRACTION_STENCIL_UNAVAILABLE, DIFFRACTION_DETECTION_UNAVAILABLE, DIFFRACTION_INVALID_DATA = 8, 16, 32


class Vec3f(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class OpticsInput(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("patches", C.c_void_p), ("directions", C.c_void_p),
                ("offsets", C.c_void_p), ("summaries", C.c_void_p), ("hits", C.c_void_p),
                ("second_input_fields", C.c_void_p), ("hit_storage_count", C.c_uint64),
                ("vertex_count", C.c_uint32), ("patch_count", C.c_uint32), ("direction_count", C.c_uint32),
                ("second_input_count", C.c_uint32), ("incident_direction", Vec3f), ("incident_basis_x", Vec3f),
                ("input_polarization", C.c_uint32), ("reserved", C.c_uint32)]


class Field32(C.Structure):
    _fields_ = [("x_real", C.c_float), ("x_imag", C.c_float), ("y_real", C.c_float), ("y_imag", C.c_float)]


class RaindropConfig(C.Structure):
    """icp_raindrop_config = rainbow::RaindropTraceConfig (116 B)."""
    _fields_ = [("coefficients", C.c_float * 8), ("inner_radius", C.c_float), ("outer_radius", C.c_float),
                ("incident_direction", Vec3f), ("incident_basis_x", Vec3f), ("incident_field", Field32),
                ("radius_mm", C.c_float), ("wavelength_nm", C.c_float), ("exterior_index", C.c_float),
                ("interior_index", C.c_float), ("grid_half_extent", C.c_float), ("reference_distance", C.c_float),
                ("outgoing_reference_distance", C.c_float), ("grid_width", C.c_uint32), ("grid_height", C.c_uint32)]


class LatticeStats(C.Structure):
    _fields_ = [("status_counts", (C.c_uint64 * 8) * 4), ("intersection_fallbacks", C.c_uint64),
                ("snell_fallbacks", C.c_uint64), ("incomplete", C.c_uint64), ("first_problem", C.c_uint64)]

    def histogram(self) -> np.ndarray:
        return np.array([[self.status_counts[f][s] for s in range(8)] for f in range(4)], dtype=np.uint64)


class FoldedConfig(C.Structure):
    _fields_ = [("relative_tolerance", C.c_double), ("maximum_panels", C.c_uint32), ("maximum_depth", C.c_uint32)]


class FoldedView(C.Structure):
    _fields_ = [("record_indices", C.c_void_p), ("records", C.c_void_p), ("patch_count", C.c_uint32),
                ("record_count", C.c_uint32)]


class FoldedStats(C.Structure):
    _fields_ = [("candidates", C.c_uint32), ("prepared", C.c_uint32), ("unresolved", C.c_uint32),
                ("branch_count", C.c_uint32), ("focal_pending_branches", C.c_uint32), ("reserved", C.c_uint32),
                ("largest_estimated_relative_error", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class FocalConfig(C.Structure):
    _fields_ = [("grid_width", C.c_uint32), ("grid_height", C.c_uint32), ("grid_half_extent", C.c_float),
                ("reserved", C.c_uint32), ("quarter_turn_offsets", C.c_uint32 * 4)]


# The lattice, patch and query records of the drop's wave stages (icp_outgoing_vertex = 
# rainbow::OutgoingVertex, icp_outgoing_patch, icp_query_hit, icp_query_summary) and the
# per-direction optical result (icp_optical_result = rainbow::PatchOpticalResult).
VERTEX_DTYPE = np.dtype([("position", "<f4", 3), ("direction", "<f4", 3), ("basis_x", "<f4", 3),
                         ("field", "<f4", 4), ("turns", "<i4"), ("fraction", "<f4"), ("status", "<u4"),
                         ("diagnostics", "<u4")])
PATCH_DTYPE = np.dtype([("vertex_indices", "<u4", 4), ("patch_id", "<u4"), ("status", "<u4"),
                        ("signed_solid_angle_sr", "<f4"), ("incident_area_drop2", "<f4")])
HIT_DTYPE = np.dtype([("compact_index", "<u4"), ("patch_id", "<u4"), ("root_index", "<u4"), ("flags", "<u4"),
                      ("u", "<f4"), ("v", "<f4"), ("t", "<f4"), ("residual", "<f4")])
SUMMARY_DTYPE = np.dtype([(k, "<u4") for k in ("candidate_count", "hit_count", "regular_hits", "refinement_hits",
                                               "boundary_hits", "flags", "first_problem_patch_id", "reserved")])
OPTICAL_DTYPE = np.dtype([("path_field", "<f8", 4), ("incoherent_s", "<f8"), ("incoherent_p", "<f8"),
                          ("path_s", "<f8"), ("path_p", "<f8")] +
                         [(k, "<u4") for k in ("hit_count", "evaluated_hits", "rejected_hits", "refinement_hits",
                                               "boundary_hits", "singular_hits", "flags", "query_flags",
                                               "first_problem_patch_id", "folded_hits")] +
                         [("path_field_second", "<f8", 4)])
AABB_DTYPE = np.dtype([(k, "<f4") for k in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z")])
FOLDED_BRANCH_DTYPE = np.dtype([("u0", "<f8"), ("u1", "<f8"), ("area_fraction", "<f8"), ("solid_angle_sr", "<f8"),
                                ("representative_u", "<f8"), ("representative_v", "<f8"), ("sign", "<i4"),
                                ("focal_flags", "<u4"), ("quarter_turns", "<u4"), ("extra_quarter_turn", "<u4")])
FOLDED_DTYPE = np.dtype([("compact_index", "<u4"), ("patch_id", "<u4"), ("flags", "<u4"), ("branch_count", "<u4"),
                         ("jacobian", "<f8", 4), ("branches", FOLDED_BRANCH_DTYPE, 4),
                         ("largest_estimated_relative_error", "<f8"), ("panels", "<u4"), ("reserved", "<u4")])


class DensityReport(C.Structure):
    _fields_ = [("maximum", C.c_double), ("invalid_values", C.c_uint64), ("incomplete", C.c_uint64),
                ("underresolved", C.c_uint64), ("first_problem", C.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


WAVE_STAGES = {"incoherent": 1, "path": 2, "focal": 3, "diffraction": 4}


class SurrogateConfig(C.Structure):
    _fields_ = [("nt", C.c_uint32), ("np", C.c_uint32), ("hidden", C.c_uint32), ("input_width", C.c_uint32),
                ("theta_frequencies", C.c_uint32), ("phi_frequencies", C.c_uint32), ("max_records", C.c_uint32),
                ("axis_harmonics", C.c_uint32), ("log_radius_mm", C.c_double * 2), ("wavelength_nm", C.c_double * 2),
                ("log_wavelength_over_radius", C.c_double * 2), ("index_center", C.c_double),
                ("index_scale", C.c_double), ("coefficient_scale", C.c_double * 8)]


class Adam(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("weight_decay", C.c_float), ("step", C.c_uint32)]


# ---------------------------------------------------------------- library loading
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_FUNCS = {
    "icp_abi_version": (C.c_uint32, []),
    "icp_kernel_launches": (C.c_ulonglong, []),
    "icp_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "icp_context_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "icp_context_destroy": (C.c_int, [_P]),
    "icp_context_synchronize": (C.c_int, [_P]),
    "icp_context_stream": (_P, [_P]),
    "icp_context_set_wait_limit": (C.c_int, [_P, C.c_uint32]),
    "icp_device_alloc": (C.c_int, [_P, C.c_size_t, C.POINTER(_P)]),
    "icp_device_free": (C.c_int, [_P, _P]),
    "icp_memcpy_h2d": (C.c_int, [_P, _P, _P, C.c_size_t]),
    "icp_memcpy_d2h": (C.c_int, [_P, _P, _P, C.c_size_t]),
    "icp_memset_d": (C.c_int, [_P, _P, C.c_int, C.c_size_t]),
    "icp_u_edges": (C.c_int, [C.c_uint32, _D]),
    "icp_ice_index": (C.c_int, [C.c_double, C.POINTER(IceState)]),
    "icp_hex_node_area": (C.c_int, [C.POINTER(HexNode), C.POINTER(Grid), _D]),
    "icp_hex_trace_bin": (C.c_int, [_P, C.POINTER(HexNode), C.POINTER(Grid), _P, _P, C.POINTER(TraceStats), _P,
                                    C.POINTER(Tuning)]),
    "icp_phase_cdf_build": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint32,
                                      C.c_uint32, C.POINTER(CdfPolicy), _P, _P, C.POINTER(CdfReport)]),
    "icp_phase_cdf_enqueue": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double,
                                        C.c_uint32, C.c_uint32, _P, _P]),
    "icp_phase_cdf_result": (C.c_int, [_P, C.POINTER(CdfPolicy), C.POINTER(CdfReport)]),
    "icp_phase_cdf_build_batch": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                            C.POINTER(CdfPolicy), _P, _P, C.POINTER(CdfReport)]),
    "icp_hex_generate": (C.c_int, [_P, C.POINTER(HexRecordArgs), C.POINTER(Orientation), C.c_uint32, _D, _D, _D,
                                   C.POINTER(RecordReport)]),
    "icp_phase_cdf_build_static": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double,
                                             C.c_uint32, C.c_uint32, C.POINTER(CdfPolicy), _P, _P,
                                             C.POINTER(CdfReport)]),
    "icp_water_index": (C.c_int, [C.c_double, C.c_double, C.c_double, _D, _D]),
    "icp_water_state": (C.c_int, [C.c_double, C.c_double, C.c_double, _D]),
    "icp_drop_shape": (C.c_int, [C.c_double, C.c_int, _D, _D, _D]),
    "icp_drop_projected_area": (C.c_int, [_D, C.c_double, _D, _D]),
    "icp_drop_frame": (C.c_int, [C.c_double, _D, _D, _D]),
    "icp_drop_diffraction_rows": (C.c_int, [_D, C.c_uint32, C.c_double, C.c_double, _D]),
    "icp_drop_sampling_area": (C.c_int, [_D, C.c_double, _D]),
    "icp_drop_trace_bin": (C.c_int, [_P, C.POINTER(DropRecordArgs), C.c_uint64, C.c_uint64, C.c_double,
                                     C.POINTER(Grid), _P, _P, C.POINTER(TraceStats)]),
    "icp_drop_generate": (C.c_int, [_P, C.POINTER(DropRecordArgs), _D, _D, _D, C.POINTER(DropReport)]),
    "icp_drop_generate_device": (C.c_int, [_P, C.POINTER(DropRecordArgs), _P, _P, _P, C.POINTER(DropReport)]),
    "icp_drop_batch_generate_device": (C.c_int, [_P, C.POINTER(DropItem), C.c_uint32, C.POINTER(BatchSettings), _P, _P,
                                                 C.POINTER(DropReport)]),
    "icp_drop_batch_generate": (C.c_int, [_P, C.POINTER(DropItem), C.c_uint32, C.POINTER(BatchSettings), _D, _D, _D,
                                          C.POINTER(DropReport)]),
    "icp_drop_batch_autotune": (C.c_int, [_P, C.POINTER(DropItem), C.c_uint32, C.POINTER(BatchSettings), _D]),
    "icp_mlp_gemm_bf16": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P, C.c_int]),
    "icp_surrogate_default_config": (C.c_int, [C.POINTER(SurrogateConfig)]),
    "icp_surrogate_parameter_count": (C.c_uint64, [C.POINTER(SurrogateConfig)]),
    "icp_surrogate_record_features": (C.c_int, [C.POINTER(SurrogateConfig), C.POINTER(DropItem), C.c_uint32, _P]),
    "icp_surrogate_cell_features": (C.c_int, [C.POINTER(SurrogateConfig), _P]),
    "icp_surrogate_inputs": (C.c_int, [_P, C.POINTER(DropItem), C.c_uint32, _P]),
    "icp_surrogate_create": (C.c_int, [_P, C.POINTER(SurrogateConfig), C.POINTER(_P)]),
    "icp_surrogate_destroy": (None, [_P]),
    "icp_surrogate_set_parameters": (C.c_int, [_P, _P, C.c_uint64]),
    "icp_surrogate_get_parameters": (C.c_int, [_P, _P, C.c_uint64]),
    "icp_surrogate_gradient": (C.c_int, [_P, C.POINTER(DropItem), C.c_uint32, _P, _P, _D]),
    "icp_surrogate_train_step": (C.c_int, [_P, C.POINTER(DropItem), C.c_uint32, _P, C.POINTER(Adam), _D]),
    "icp_surrogate_predict": (C.c_int, [_P, C.POINTER(DropItem), C.c_uint32, _P]),
    "icp_surrogate_generate": (C.c_int, [_P, C.POINTER(DropItem), C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.POINTER(CdfPolicy), _P, _P, C.POINTER(CdfReport)]),
    "icp_surrogate_targets": (C.c_int, [_P, _P, _P, C.c_uint32, _P]),
    "icp_atlas_area_rule": (C.c_int, [C.c_double, C.c_double, _D, C.c_uint32, C.POINTER(AtlasRay), C.c_uint64,
                                      C.POINTER(C.c_uint64)]),
    "icp_atlas_incident_node": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.POINTER(AtlasIncident)]),
    "icp_atlas_trace_node": (C.c_int, [_P, C.POINTER(AtlasSettings), C.c_uint32, C.c_uint32, _P,
                                       C.POINTER(AtlasNodeReport)]),
    "icp_atlas_coupling": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, _D, _P, _P,
                                     C.c_uint64, _D, C.c_double, C.c_int, _P, _D]),
    "icp_atlas_compose": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P, _P]),
    "icp_patch_build": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.c_float, _P, _P, _P, C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint64)]),
    "icp_raindrop_config_make": (C.c_int, [C.c_float, C.c_int, C.POINTER(C.c_float), C.c_float, C.c_float,
                                           C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.POINTER(RaindropConfig)]),
    "icp_lattice_trace": (C.c_int, [_P, C.POINTER(RaindropConfig), _P, _P, C.POINTER(LatticeStats)]),
    "icp_query_directions": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                       C.POINTER(C.c_float)]),
    "icp_patch_query": (C.c_int, [_P, _P, C.c_uint32, _P, _P, C.c_uint32, _P, C.c_uint32, _P, _P, _P, C.c_uint64,
                                  C.POINTER(C.c_uint64)]),
    "icp_patch_optics": (C.c_int, [_P, C.POINTER(OpticsInput), _P, C.POINTER(FocalConfig), _P]),
    "icp_patch_optics_folded": (C.c_int, [_P, C.POINTER(OpticsInput), _P, C.POINTER(FocalConfig), _P,
                                          C.POINTER(FoldedView)]),
    "icp_folded_prepare": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(FocalConfig),
                                     C.POINTER(FoldedConfig), _P, _P, C.c_uint32, C.POINTER(C.c_uint32),
                                     C.POINTER(FoldedStats)]),
    "icp_stage_density": (C.c_int, [_P, C.c_uint32, _P, _P, _P, C.c_uint64, _P, C.POINTER(DensityReport)]),
    "icp_rainbow_table_sigma": (C.c_int, [C.c_float, _D]),
    "icp_rainbow_detect": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.POINTER(DiffractionConfig), _P]),
    "icp_rainbow_filter": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_uint32, C.POINTER(DiffractionConfig), _P, _P,
                                     C.POINTER(DiffractionStats)]),
    "icp_rainbow_diffraction": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.POINTER(DiffractionConfig), _P, _P, _P,
                                          C.POINTER(DiffractionStats)]),
}


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python ice_crystal_phase_b200/build.py` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _FUNCS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


LIB = _load()


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    LIB.icp_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != ICP_OK:
        raise _ERRORS.get(status, IcpError)(status, last_error())


def exported_symbols() -> list[str]:
    return list(_FUNCS)


def kernel_launches() -> int:
    """CUDA kernels launched by libicp_b200 in this process."""
    return int(LIB.icp_kernel_launches())


# ---------------------------------------------------------------- host-side values
def u_edges(nt: int) -> np.ndarray:
    e = np.empty(nt + 1)
    check(LIB.icp_u_edges(nt, e.ctypes.data_as(_D)))
    return e


def evaluate_ice_optics(vacuum_wavelength_nm: float) -> IceState:
    """Refractive index of ice Ih (Warren & Brandt 2008) at a vacuum wavelength in 200..1100 nm
    (evaluate_ice_wb2008, hex_atlas/src/ice_optics.cpp:13-30): the interior index of a prism
    record at that wavelength.  Raises InvalidArgument outside the table."""
    st = IceState()
    check(LIB.icp_ice_index(float(vacuum_wavelength_nm), C.byref(st)))
    return st


def atlas_area_rule(circumradius_mm: float, length_mm: float, ki, subdivisions: int):
    """Projected-area quadrature of the prism lit from ki (atlas::make_area_rule,
    hex_atlas/src/atlas.cpp:11-51): (faces[n], points[n][3] in units of the circumradius,
    weights_mm2[n])."""
    k = (C.c_double * 3)(*map(float, ki))
    n = C.c_uint64()
    check(LIB.icp_atlas_area_rule(float(circumradius_mm), float(length_mm), k, int(subdivisions), None, 0,
                                  C.byref(n)))
    rays = (AtlasRay * max(1, n.value))()
    check(LIB.icp_atlas_area_rule(float(circumradius_mm), float(length_mm), k, int(subdivisions), rays, n.value,
                                  C.byref(n)))
    a = np.frombuffer(rays, dtype=np.dtype([("face", "<u4"), ("reserved", "<u4"), ("x", "<f8"), ("y", "<f8"),
                                            ("z", "<f8"), ("w", "<f8")]), count=n.value)
    return a["face"].copy(), np.stack([a["x"], a["y"], a["z"]], axis=1), a["w"].copy()


def atlas_incident_node(theta_intervals: int, phi_intervals: int, i: int, j: int) -> AtlasIncident:
    """Incident node (i, j) of the symmetry domain (the frame part of atlas::make_node)."""
    out = AtlasIncident()
    check(LIB.icp_atlas_incident_node(int(theta_intervals), int(phi_intervals), int(i), int(j), C.byref(out)))
    return out


def _normalize(a):
    s = max(abs(a[0]), abs(a[1]), abs(a[2]))
    if not (s > 0) or not math.isfinite(s):
        raise ValueError("Invalid incident direction.")
    a = [a[0] / s, a[1] / s, a[2] / s]
    n = math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
    return [a[0] / n, a[1] / n, a[2] / n]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def make_frame(k) -> tuple[list, list, list]:
    """Transverse frame of a direction (hex_trace/include/ice_crystal/math.hpp:61-69)."""
    k = _normalize([float(x) for x in k])
    ax, ay, az = abs(k[0]), abs(k[1]), abs(k[2])
    a = [1.0, 0.0, 0.0] if (ax <= ay and ax <= az) else ([0.0, 1.0, 0.0] if ay <= az else [0.0, 0.0, 1.0])
    d = k[0] * a[0] + k[1] * a[1] + k[2] * a[2]
    e0 = _normalize([a[i] - k[i] * d for i in range(3)])
    e1 = _normalize(_cross(k, e0))
    return k, e0, e1


@dataclass
class PhaseGrid:
    nt: int
    np: int
    ki: list
    e0: list
    e1: list
    edges: np.ndarray

    def abi(self) -> Grid:
        g = Grid()
        g.nt, g.np = self.nt, self.np
        for i in range(3):
            g.ki[i], g.e0[i], g.e1[i] = self.ki[i], self.e0[i], self.e1[i]
        return g

    def sampling_frame_columns(self) -> list:
        return [[self.e0[r], self.e1[r], self.ki[r]] for r in range(3)]


def make_phase_grid(nt: int, np_: int, ki) -> PhaseGrid:
    if not nt or not np_ or nt * np_ > 0xFFFFFFFF or nt > 32 * 65535 or np_ > 0x7FFFFFFF:
        raise ValueError("Unsupported phase grid dimensions.")
    k, e0, e1 = make_frame(ki)
    return PhaseGrid(nt, np_, k, e0, e1, u_edges(nt))


def rotation_from_quaternion(w: float, x: float, y: float, z: float) -> list:
    """Column-major body->ensemble rotation (hex_phase/src/phase_table.cpp:11-21)."""
    n = w * w + x * x + y * y + z * z
    if not math.isfinite(n) or abs(n - 1) > 2e-12:
        raise ValueError("Quaternion must be unit length (w,x,y,z).")
    k = 1 / math.sqrt(n)
    w, x, y, z = w * k, x * k, y * k, z * k
    return [1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y),
            2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x),
            2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)]


@dataclass
class OrientationNode:
    quaternion: tuple
    weight: float
    samples: int
    seed: int


@dataclass
class OrientationPlan:
    nodes: list
    total_samples: int
    input_weight_sum: float
    source_sha256: str


def parse_orientation_plan(text: str | bytes) -> OrientationPlan:
    """qw,qx,qy,qz,weight,samples,seed CSV (hex_phase/src/orientation_plan.cpp:69-120)."""
    raw = text.encode() if isinstance(text, str) else text
    sha = hashlib.sha256(raw).hexdigest()
    nodes, header, total = [], False, 0
    s, c = 0.0, 0.0
    for number, line in enumerate(raw.decode().split("\n"), 1):
        line = line.strip(" \t\r")
        if not line or line.startswith("#"):
            continue
        try:
            if not header:
                if line != "qw,qx,qy,qz,weight,samples,seed":
                    raise ValueError("Expected CSV header qw,qx,qy,qz,weight,samples,seed.")
                header = True
                continue
            cols = line.split(",")
            if len(cols) != 7:
                raise ValueError("Expected seven CSV fields.")
            q = tuple(float(x.strip(" \t\r")) for x in cols[:4])
            rotation_from_quaternion(*q)
            weight, samples, seed = float(cols[4]), int(cols[5]), int(cols[6])
            if not math.isfinite(weight) or not weight > 0 or samples <= 0:
                raise ValueError("Weights and sample counts must be positive.")
            if samples > 2 ** 64 - 1 - total or seed < 0 or seed >= 2 ** 64:
                raise OverflowError("Planned sample count overflows.")
            total += samples
            y = weight - c
            t = s + y
            c = (t - s) - y
            s = t
            nodes.append(OrientationNode(q, weight, samples, seed))
        except (ValueError, OverflowError) as e:
            raise ValueError(f"Orientation CSV line {number}: {e}") from None
    if not header or not nodes or not math.isfinite(s) or abs(s - 1) > 2e-12:
        raise ValueError("Orientation number-probability weights must sum to one (within 2e-12).")
    for n in nodes:
        n.weight /= s
    return OrientationPlan(nodes, total, s, sha)


# ---------------------------------------------------------------- device context
class Context:
    """One CUDA device and one non-blocking stream (rainbow::CudaContext, src/cuda_driver.cpp:148-215)."""

    def __init__(self, device: int = 0):
        h = _P()
        check(LIB.icp_context_create(device, C.byref(h)))
        self.handle = h

    def close(self) -> None:
        if self.handle:
            LIB.icp_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceArray:
    """Context-owned device allocation of float64 (or raw bytes) for FFI-style callers."""

    def __init__(self, ctx: Context, count: int, dtype=np.float64):
        self.ctx, self.dtype, self.count = ctx, np.dtype(dtype), count
        self.nbytes = max(1, count * self.dtype.itemsize)
        p = _P()
        check(LIB.icp_device_alloc(ctx.handle, self.nbytes, C.byref(p)))
        self.ptr = p

    def upload(self, host: np.ndarray) -> "DeviceArray":
        a = np.ascontiguousarray(host, dtype=self.dtype)
        assert a.size == self.count
        check(LIB.icp_memcpy_h2d(self.ctx.handle, self.ptr, a.ctypes.data_as(_P), a.nbytes))
        return self

    def download(self) -> np.ndarray:
        out = np.empty(self.count, dtype=self.dtype)
        check(LIB.icp_memcpy_d2h(self.ctx.handle, out.ctypes.data_as(_P), self.ptr, out.nbytes))
        return out

    def zero(self) -> "DeviceArray":
        check(LIB.icp_memset_d(self.ctx.handle, self.ptr, 0, self.nbytes))
        return self

    def free(self) -> None:
        if self.ptr:
            LIB.icp_device_free(self.ctx.handle, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PhaseMassAccumulatorCuda:
    """FP64 cell-mass histogram fed by the fused hex trace+bin kernel.

    ``add_hex_node`` replaces HexPrismTracer::trace + PhaseMassAccumulatorCuda::add for one
    orientation node (all its ray batches in one launch); ``masses`` returns the cell masses
    with the pole caps spread over the end rows (PhaseMassAccumulator::masses).
    """

    def __init__(self, ctx: Context, grid: PhaseGrid):
        self.ctx, self.grid = ctx, grid
        self.edges = DeviceArray(ctx, grid.nt + 1).upload(grid.edges)
        self.mass = DeviceArray(ctx, grid.nt * grid.np).zero()
        self.stats = TraceStats()
        self.forward = 0.0
        self.backward = 0.0
        self.escaped_area = 0.0
        self.unresolved_area = 0.0
        self.point_axial = 0.0

    def add_hex_node(self, prism: tuple[float, float], quaternion, weight: float, samples: int, seed: int,
                     interior_index: float, exterior_index: float = 1.0, max_internal_hits: int = 1024,
                     tail_tolerance: float = 1e-12, precision: int = ICP_FP32, balance_tolerance: float | None = None,
                     first: int = 0, count: int | None = None, tuning: Tuning | None = None,
                     batch_size: int = 4096) -> TraceStats:
        n = HexNode()
        n.circumradius_mm, n.length_mm = prism
        for i, v in enumerate(rotation_from_quaternion(*quaternion)):
            n.rotation[i] = v
        n.exterior_index, n.interior_index = exterior_index, interior_index
        n.tail_tolerance = tail_tolerance
        n.balance_tolerance = 1e-10 if balance_tolerance is None else balance_tolerance
        n.seed, n.total_samples, n.first_sample = seed, samples, first
        n.sample_count = samples - first if count is None else count
        n.max_internal_hits, n.batch_size, n.precision = max_internal_hits, batch_size, precision
        g = self.grid.abi()
        area = C.c_double()
        n.area_weight = 1.0
        check(LIB.icp_hex_node_area(C.byref(n), C.byref(g), C.byref(area)))
        n.area_weight = weight * area.value / float(samples)
        s = TraceStats()
        check(LIB.icp_hex_trace_bin(self.ctx.handle, C.byref(n), C.byref(g), self.edges.ptr, self.mass.ptr, C.byref(s),
                                    None, C.byref(tuning) if tuning else None))
        self.forward += n.area_weight * s.forward_pole
        self.backward += n.area_weight * s.backward_pole
        self.escaped_area += n.area_weight * s.escaped
        self.unresolved_area += n.area_weight * s.unresolved
        self.point_axial += n.area_weight * s.point_axial
        for k, _ in TraceStats._fields_:
            if k == "status_counts":
                for i in range(8):
                    self.stats.status_counts[i] += s.status_counts[i]
            elif k.startswith("max_"):
                setattr(self.stats, k, max(getattr(self.stats, k), getattr(s, k)))
            else:
                setattr(self.stats, k, getattr(self.stats, k) + getattr(s, k))
        return s

    def cell_mass(self) -> np.ndarray:
        """Raw cell masses (without pole caps), theta-major."""
        return self.mass.download()

    def masses(self) -> np.ndarray:
        m = self.cell_mass().reshape(self.grid.nt, self.grid.np)
        m[0] += self.forward / self.grid.np
        m[-1] += self.backward / self.grid.np
        return m.reshape(-1)


@dataclass
class CdfResult:
    phi: np.ndarray
    theta: np.ndarray
    u_edges: np.ndarray
    report: dict


class PhaseCdf:
    """Stored CDF builder (rainbow::PhaseCdf::build + build_host_cdf arithmetic)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def build(self, values, nt: int, np_: int, ct: int | None = None, cp: int | None = None,
              forward: float = 0.0, backward: float = 0.0, density: bool = False, max_l1_error: float = 1e-10,
              max_lost_mass: float = 1e-12, max_coarsening_tv: float = 1.0) -> CdfResult:
        ct, cp = ct or nt, cp or np_
        if isinstance(values, DeviceArray):
            dv = values
        else:
            dv = DeviceArray(self.ctx, nt * np_).upload(np.asarray(values, dtype=np.float64).reshape(-1))
        phi = DeviceArray(self.ctx, cp + 1)
        theta = DeviceArray(self.ctx, cp * (ct + 1))
        pol = CdfPolicy(max_l1_error, max_lost_mass, max_coarsening_tv)
        rep = CdfReport()
        check(LIB.icp_phase_cdf_build(self.ctx.handle, dv.ptr, 1 if density else 0, nt, np_, forward, backward, ct, cp,
                                      C.byref(pol), phi.ptr, theta.ptr, C.byref(rep)))
        edges = u_edges(nt)[:: nt // ct].copy()
        return CdfResult(phi.download(), theta.download().reshape(cp, ct + 1), edges, rep.as_dict())


@dataclass
class HexRecordResult:
    phi: np.ndarray
    theta: np.ndarray
    u_edges: np.ndarray
    report: RecordReport
    grid: PhaseGrid


def generate_hex_record(ctx: Context, circumradius_mm: float, length_mm: float, ki, interior_index: float,
                        nt: int, np_: int, plan: OrientationPlan, ct: int | None = None, cp: int | None = None,
                        exterior_index: float = 1.0, max_internal_hits: int = 1024, tail_tolerance: float = 1e-12,
                        precision: int = ICP_FP32, balance_tolerance: float | None = None, batch_size: int = 4096,
                        max_output_records: int = 0, max_l1_error: float = 1e-10, max_lost_mass: float = 1e-12,
                        max_coarsening_tv: float = 1.0, tuning: Tuning | None = None) -> HexRecordResult:
    """One hex record through the host-buffer C-ABI entry (icp_hex_generate)."""
    ct, cp = ct or nt, cp or np_
    r = HexRecordArgs()
    r.circumradius_mm, r.length_mm = circumradius_mm, length_mm
    for i in range(3):
        r.ki[i] = float(ki[i])
    r.exterior_index, r.interior_index = exterior_index, interior_index
    r.tail_tolerance = tail_tolerance
    r.balance_tolerance = 1e-10 if balance_tolerance is None else balance_tolerance
    r.nt, r.np, r.ct, r.cp = nt, np_, ct, cp
    r.max_internal_hits, r.batch_size, r.max_output_records = max_internal_hits, batch_size, max_output_records
    r.precision = precision
    r.policy = CdfPolicy(max_l1_error, max_lost_mass, max_coarsening_tv)
    if tuning:
        r.tuning = tuning
    nodes = (Orientation * len(plan.nodes))()
    for i, n in enumerate(plan.nodes):
        for j in range(4):
            nodes[i].quaternion[j] = n.quaternion[j]
        nodes[i].weight, nodes[i].samples, nodes[i].seed = n.weight, n.samples, n.seed
    phi = np.empty(cp + 1)
    theta = np.empty(cp * (ct + 1))
    u = np.empty(ct + 1)
    rep = RecordReport()
    check(LIB.icp_hex_generate(ctx.handle, C.byref(r), nodes, len(plan.nodes), phi.ctypes.data_as(_D),
                               theta.ctypes.data_as(_D), u.ctypes.data_as(_D), C.byref(rep)))
    return HexRecordResult(phi, theta.reshape(cp, ct + 1), u, rep, make_phase_grid(nt, np_, ki))



# ---------------------------------------------------------------- water drops
@dataclass
class WaterOpticalState:
    refractive_index: float
    density_kg_m3: float
    temperature_kelvin: float
    pressure_pascal: float
    density_pressure_residual_pascal: float = 0.0
    density_bracket_width_kg_m3: float = 0.0


def evaluate_water_optics(vacuum_wavelength_nm: float, temperature_celsius: float = 20.0,
                          pressure_pascal: float = 101325.0) -> WaterOpticalState:
    """IAPWS R9-97 real index of liquid water with its IAPWS-95 density (evaluate_water_optics);
    bounded to 200..1100 nm, 0..60 C, 50 kPa..100 MPa."""
    w = (C.c_double * 6)()
    check(LIB.icp_water_state(vacuum_wavelength_nm, temperature_celsius, pressure_pascal, w))
    return WaterOpticalState(w[5], w[2], w[0], w[1], w[3], w[4])


@dataclass
class RaindropShape:
    """r/a = 1 + sum_n coefficients[n] cos(n chi), chi from the particle's -y axis."""
    coefficients: list
    inner_radius: float
    outer_radius: float

    @staticmethod
    def make(radius_mm: float, sphere: bool = False) -> "RaindropShape":
        c = (C.c_double * 8)()
        lo, hi = C.c_double(), C.c_double()
        check(LIB.icp_drop_shape(radius_mm, int(sphere), c, C.byref(lo), C.byref(hi)))
        return RaindropShape(list(c), lo.value, hi.value)


def _c8(coefficients) -> C.Array:
    c = [float(x) for x in coefficients]
    if len(c) > 8:
        raise ValueError("At most eight shape coefficients.")
    return (C.c_double * 8)(*(c + [0.0] * (8 - len(c))))


def compute_projected_area(coefficients, radius_mm: float, incident_propagation) -> float:
    """Projected area (mm^2) of the convex drop along the incident direction, binary64 on the CPU."""
    k = (C.c_double * 3)(*map(float, incident_propagation))
    a = C.c_double()
    check(LIB.icp_drop_projected_area(_c8(coefficients), radius_mm, k, C.byref(a)))
    return a.value


def drop_frame(inclination_deg: float) -> tuple[list, list, list]:
    """ki = (cos a, -sin a, 0) and the frame of the stored CDF (sampling_frame_columns)."""
    k, e0, e1 = (C.c_double * 3)(), (C.c_double * 3)(), (C.c_double * 3)()
    check(LIB.icp_drop_frame(inclination_deg, k, e0, e1))
    return list(k), list(e0), list(e1)


def make_drop_grid(nt: int, np_: int, inclination_deg: float) -> PhaseGrid:
    if not nt or not np_ or nt * np_ > 0xFFFFFFFF:
        raise ValueError("Unsupported phase grid dimensions.")
    k, e0, e1 = drop_frame(inclination_deg)
    return PhaseGrid(nt, np_, k, e0, e1, u_edges(nt))


def sampling_area(coefficients, radius_mm: float) -> float:
    a = C.c_double()
    check(LIB.icp_drop_sampling_area(_c8(coefficients), radius_mm, C.byref(a)))
    return a.value


def diffraction_rows(edges: np.ndarray, area_mm2: float, wavelength_nm: float) -> np.ndarray:
    e = np.ascontiguousarray(edges, dtype=np.float64)
    rows = np.empty(e.size - 1)
    check(LIB.icp_drop_diffraction_rows(e.ctypes.data_as(_D), e.size - 1, area_mm2, wavelength_nm,
                                        rows.ctypes.data_as(_D)))
    return rows


def _drop_args(coefficients, radius_mm, inclination_deg, interior_index, rays, seed, nt, np_, ct, cp,
               exterior_index, max_internal_hits, tail_tolerance, precision, balance_tolerance, wavelength_nm,
               diffraction, max_l1_error=1e-10, max_lost_mass=1e-12, max_coarsening_tv=1.0, tuning=None):
    r = DropRecordArgs()
    r.radius_mm = radius_mm
    r.coefficients = _c8(coefficients)
    r.inclination_deg = inclination_deg
    r.exterior_index, r.interior_index, r.wavelength_nm = exterior_index, interior_index, wavelength_nm
    r.tail_tolerance = tail_tolerance
    r.balance_tolerance = 1e-10 if balance_tolerance is None else balance_tolerance
    r.nt, r.np, r.ct, r.cp = nt, np_, ct, cp
    r.max_internal_hits, r.precision = max_internal_hits, precision
    r.rays, r.seed, r.diffraction = rays, seed, int(bool(diffraction))
    r.policy = CdfPolicy(max_l1_error, max_lost_mass, max_coarsening_tv)
    if tuning:
        r.tuning = tuning
    return r


def _add_drop(self, coefficients, radius_mm: float, interior_index: float, rays: int, seed: int,
              inclination_deg: float, exterior_index: float = 1.0, max_internal_hits: int = 1024,
              tail_tolerance: float = 1e-12, precision: int = ICP_FP32, first: int = 0, count: int | None = None,
              tuning: Tuning | None = None, balance_tolerance: float | None = None) -> TraceStats:
    """Traces rays [first, first+count) of one drop (sampled on its bounding disk) into the
    histogram; the grid must be the drop frame's (make_drop_grid)."""
    r = _drop_args(coefficients, radius_mm, inclination_deg, interior_index, rays, seed, self.grid.nt, self.grid.np,
                   self.grid.nt, self.grid.np, exterior_index, max_internal_hits, tail_tolerance, precision,
                   balance_tolerance, 0.0, False, tuning=tuning)
    weight = sampling_area(coefficients, radius_mm) / float(rays)
    g = self.grid.abi()
    s = TraceStats()
    count = rays - first if count is None else count
    check(LIB.icp_drop_trace_bin(self.ctx.handle, C.byref(r), first, count, weight, C.byref(g), self.edges.ptr,
                                 self.mass.ptr, C.byref(s)))
    self.forward += weight * s.forward_pole
    self.backward += weight * s.backward_pole
    self.escaped_area += weight * s.escaped
    self.unresolved_area += weight * s.unresolved
    self.point_axial += weight * s.point_axial
    self.incident_area = getattr(self, "incident_area", 0.0) + weight * (s.rays - s.missed)
    for k, _ in TraceStats._fields_:
        if k == "status_counts":
            for i in range(8):
                self.stats.status_counts[i] += s.status_counts[i]
        elif k.startswith("max_"):
            setattr(self.stats, k, max(getattr(self.stats, k), getattr(s, k)))
        else:
            setattr(self.stats, k, getattr(self.stats, k) + getattr(s, k))
    return s


PhaseMassAccumulatorCuda.add_drop = _add_drop


@dataclass
class DropRecordResult:
    phi: np.ndarray
    theta: np.ndarray
    u_edges: np.ndarray
    report: DropReport
    grid: PhaseGrid


def generate_drop_record(ctx: Context, coefficients, radius_mm: float, interior_index: float, nt: int, np_: int,
                         rays: int, seed: int = 12345, inclination_deg: float = 20.0, ct: int | None = None,
                         cp: int | None = None, exterior_index: float = 1.0, max_internal_hits: int = 1024,
                         tail_tolerance: float = 1e-12, precision: int = ICP_FP32, wavelength_nm: float = 0.0,
                         diffraction: bool = False, balance_tolerance: float | None = None,
                         max_l1_error: float = 1e-10, max_lost_mass: float = 1e-12, max_coarsening_tv: float = 1.0,
                         tuning: Tuning | None = None) -> DropRecordResult:
    """One drop record through the host-buffer C-ABI entry (icp_drop_generate)."""
    ct, cp = ct or nt, cp or np_
    r = _drop_args(coefficients, radius_mm, inclination_deg, interior_index, rays, seed, nt, np_, ct, cp,
                   exterior_index, max_internal_hits, tail_tolerance, precision, balance_tolerance, wavelength_nm,
                   diffraction, max_l1_error, max_lost_mass, max_coarsening_tv, tuning)
    phi = np.empty(cp + 1)
    theta = np.empty(cp * (ct + 1))
    u = np.empty(ct + 1)
    rep = DropReport()
    check(LIB.icp_drop_generate(ctx.handle, C.byref(r), phi.ctypes.data_as(_D), theta.ctypes.data_as(_D),
                                u.ctypes.data_as(_D), C.byref(rep)))
    return DropRecordResult(phi, theta.reshape(cp, ct + 1), u, rep, make_drop_grid(nt, np_, inclination_deg))


# ---------------------------------------------------------------- batched drop records
@dataclass
class DropSpec:
    """One record of a batch (the per-record parameters of a rainbow_generate run)."""
    coefficients: list
    radius_mm: float
    interior_index: float
    rays: int
    seed: int = 12345
    inclination_deg: float = 20.0
    wavelength_nm: float = 0.0
    diffraction: bool = False


def batch_settings(nt: int, np_: int, ct: int | None = None, cp: int | None = None, max_internal_hits: int = 1024,
                   precision: int = ICP_FP32, exterior_index: float = 1.0, tail_tolerance: float = 1e-12,
                   balance_tolerance: float = 1e-10, max_l1_error: float = 1e-10, max_lost_mass: float = 1e-12,
                   max_coarsening_tv: float = 1.0, block_threads: int = 0, blocks_per_sm: int = 0,
                   chunk_rays: int = 0, use_graph: bool = True) -> BatchSettings:
    s = BatchSettings()
    s.nt, s.np, s.ct, s.cp = nt, np_, ct or nt, cp or np_
    s.max_internal_hits, s.precision = max_internal_hits, precision
    s.exterior_index, s.tail_tolerance, s.balance_tolerance = exterior_index, tail_tolerance, balance_tolerance
    s.policy = CdfPolicy(max_l1_error, max_lost_mass, max_coarsening_tv)
    s.block_threads, s.blocks_per_sm, s.chunk_rays, s.use_graph = block_threads, blocks_per_sm, chunk_rays, int(use_graph)
    return s


# icp_drop_item as a NumPy record with the ctypes structure's own offsets, so that a batch of
# items is filled column by column rather than one ctypes field at a time
_DROP_ITEM_DTYPE = np.dtype({
    "names": ["radius_mm", "coefficients", "inclination_deg", "interior_index", "wavelength_nm", "rays", "seed",
              "diffraction"],
    "formats": ["<f8", ("<f8", 8), "<f8", "<f8", "<f8", "<u8", "<u8", "<u4"],
    "offsets": [getattr(DropItem, f).offset for f in ("radius_mm", "coefficients", "inclination_deg", "interior_index",
                                                      "wavelength_nm", "rays", "seed", "diffraction")],
    "itemsize": C.sizeof(DropItem)})


def _items(specs) -> C.Array:
    n = len(specs)
    arr = (DropItem * n)()
    if not n:
        return arr
    v = np.frombuffer(arr, dtype=_DROP_ITEM_DTYPE, count=n)
    coeffs = [[float(x) for x in sp.coefficients] for sp in specs]
    if any(len(c) > 8 for c in coeffs):
        raise ValueError("At most eight shape coefficients.")
    v["coefficients"] = [c + [0.0] * (8 - len(c)) for c in coeffs]
    v["radius_mm"] = [sp.radius_mm for sp in specs]
    v["inclination_deg"] = [sp.inclination_deg for sp in specs]
    v["interior_index"] = [sp.interior_index for sp in specs]
    v["wavelength_nm"] = [sp.wavelength_nm for sp in specs]
    v["rays"] = [int(sp.rays) for sp in specs]
    v["seed"] = [int(sp.seed) for sp in specs]
    v["diffraction"] = [int(bool(sp.diffraction)) for sp in specs]
    return arr


@dataclass
class DropBatchResult:
    phi: np.ndarray          # (records, cp + 1)
    theta: np.ndarray        # (records, cp, ct + 1)
    u_edges: np.ndarray
    reports: list


def generate_drop_batch(ctx: Context, specs: list, settings: BatchSettings) -> DropBatchResult:
    """Many drop records in one persistent launch (icp_drop_batch_generate, host outputs)."""
    n = len(specs)
    items = _items(specs)
    phi = np.empty(n * (settings.cp + 1))
    theta = np.empty(n * settings.cp * (settings.ct + 1))
    u = np.empty(settings.ct + 1)
    reps = (DropReport * n)()
    check(LIB.icp_drop_batch_generate(ctx.handle, items, n, C.byref(settings), phi.ctypes.data_as(_D),
                                      theta.ctypes.data_as(_D), u.ctypes.data_as(_D), reps))
    return DropBatchResult(phi.reshape(n, settings.cp + 1), theta.reshape(n, settings.cp, settings.ct + 1), u,
                           list(reps))


def batched_record_specs(count: int = 256, seed: int = 20260101, rays_max: float = 6e7, rays_min: float = 1e6,
                         diffraction: bool = True, rays_scale: float = 1.0, radius_range: tuple = (0.1, 3.0)) -> list:
    """Drop records of the batched workload: radius log-uniform in [0.1, 3] mm (radius_range),
    wavelength uniform in [400, 700] nm, inclination uniform in [-90, 90] deg, Table-I shapes,
    water at 20 C, rays proportional to the projected area (rays_max for the area of a 3 mm
    disk), clipped to [rays_min, rays_max] and then multiplied by rays_scale."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(count):
        radius = float(np.exp(rng.uniform(np.log(radius_range[0]), np.log(radius_range[1]))))
        lam = float(rng.uniform(400.0, 700.0))
        incl = float(rng.uniform(-90.0, 90.0))
        r32 = float(np.float32(radius))
        shape = RaindropShape.make(r32).coefficients
        n = float(np.float32(evaluate_water_optics(lam).refractive_index))
        area = compute_projected_area(shape, r32, drop_frame(incl)[0])
        rays = int(min(rays_max, max(rays_min, round(rays_max * area / (math.pi * 9.0)))))
        specs.append(DropSpec(shape, r32, n, max(1, int(round(rays * rays_scale))),
                              seed=int(rng.integers(1, 2**63)), inclination_deg=incl, wavelength_nm=lam,
                              diffraction=diffraction))
    return specs


def autotune_drop_batch(ctx: Context, specs: list, settings: BatchSettings) -> float:
    """Times candidate block and chunk sizes on a bounded sample of the batch; stores the best
    in ``settings`` (and in the context for later batches).  Returns the best rays/s."""
    best = C.c_double()
    check(LIB.icp_drop_batch_autotune(ctx.handle, _items(specs), len(specs), C.byref(settings), C.byref(best)))
    return best.value


# ---------------------------------------------------------------- surrogate building blocks
def mlp_gemm_bf16(ctx: Context, a_ptr: int, b_ptr: int, m: int, n: int, k: int, c_ptr: int, accumulate: bool = False,
                  split_k: int = 1) -> None:
    """C[m x n] (FP32, device) = / += A[m x k] * B[n x k]^T (BF16, device, K contiguous) on the
    tensor cores (icp_mlp_gemm_bf16)."""
    check(LIB.icp_mlp_gemm_bf16(ctx.handle, C.c_void_p(a_ptr), C.c_void_p(b_ptr), m, n, k, split_k, C.c_void_p(c_ptr),
                                int(accumulate)))


# ---------------------------------------------------------------- learned surrogate
def surrogate_config(**overrides) -> SurrogateConfig:
    """Default surrogate configuration (256 x 512 cells, 3 x 256 hidden, input width 128) with
    field overrides; array fields take sequences."""
    cfg = SurrogateConfig()
    check(LIB.icp_surrogate_default_config(C.byref(cfg)))
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise ValueError(f"unknown surrogate config field {k!r}")
        if isinstance(v, (list, tuple)):
            arr = getattr(cfg, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(cfg, k, v)
    return cfg


def surrogate_parameter_count(cfg: SurrogateConfig) -> int:
    n = int(LIB.icp_surrogate_parameter_count(C.byref(cfg)))
    if n == 0:
        raise InvalidArgument(ICP_ERR_INVALID_ARGUMENT, "Invalid surrogate configuration.")
    return n


def surrogate_record_features(cfg: SurrogateConfig, specs) -> np.ndarray:
    """16 BF16 feature bits per record (uint16), computed by the library on the host."""
    items = _items(specs)
    out = np.zeros((len(specs), 16), dtype=np.uint16)
    check(LIB.icp_surrogate_record_features(C.byref(cfg), items, len(specs), C.c_void_p(out.ctypes.data)))
    return out


def surrogate_cell_features(cfg: SurrogateConfig) -> np.ndarray:
    """The cell table: nt*np rows x (input_width - 16) BF16 bits (uint16), theta-major cells."""
    out = np.zeros((cfg.nt * cfg.np, cfg.input_width - 16), dtype=np.uint16)
    check(LIB.icp_surrogate_cell_features(C.byref(cfg), C.c_void_p(out.ctypes.data)))
    return out


class Surrogate:
    """Handle of one surrogate network on a context (icp_surrogate_*).  Device arrays are passed
    as integer pointers (e.g. torch's data_ptr())."""

    def __init__(self, ctx: Context, cfg: SurrogateConfig):
        self.ctx, self.cfg = ctx, cfg
        self.n_params = surrogate_parameter_count(cfg)
        self.cells = cfg.nt * cfg.np
        h = _P()
        check(LIB.icp_surrogate_create(ctx.handle, C.byref(cfg), C.byref(h)))
        self.handle = h

    def close(self) -> None:
        if self.handle:
            LIB.icp_surrogate_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_parameters(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        check(LIB.icp_surrogate_set_parameters(self.handle, C.c_void_p(p.ctypes.data), p.size))

    def parameters(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        check(LIB.icp_surrogate_get_parameters(self.handle, C.c_void_p(p.ctypes.data), p.size))
        return p

    def gradient(self, specs, target_ptr: int, with_grad: bool = True) -> tuple[float, np.ndarray | None]:
        g = np.zeros(self.n_params, dtype=np.float32) if with_grad else None
        loss = C.c_double()
        check(LIB.icp_surrogate_gradient(self.handle, _items(specs), len(specs), C.c_void_p(target_ptr),
                                         C.c_void_p(g.ctypes.data) if with_grad else None, C.byref(loss)))
        return loss.value, g

    def train_step(self, specs, target_ptr: int, opt: Adam) -> float:
        loss = C.c_double()
        check(LIB.icp_surrogate_train_step(self.handle, _items(specs), len(specs), C.c_void_p(target_ptr),
                                           C.byref(opt), C.byref(loss)))
        return loss.value

    def inputs(self, specs) -> np.ndarray:
        """The device's input rows for these records: uint16 BF16 bits [len(specs) * cells, width]."""
        out = np.zeros((len(specs) * self.cells, self.cfg.input_width), dtype=np.uint16)
        check(LIB.icp_surrogate_inputs(self.handle, _items(specs), len(specs), C.c_void_p(out.ctypes.data)))
        return out

    def predict(self, specs, logits_ptr: int) -> None:
        check(LIB.icp_surrogate_predict(self.handle, _items(specs), len(specs), C.c_void_p(logits_ptr)))

    def generate(self, specs, ct: int, cp: int, phi_ptr: int, theta_ptr: int, policy: CdfPolicy | None = None,
                 raise_on_audit: bool = True) -> list:
        """Records from the prediction (device phi / theta); returns the per-record CDF reports."""
        pol = policy or CdfPolicy(1e-10, 1e-12, 1.0)
        reps = (CdfReport * len(specs))()
        st = LIB.icp_surrogate_generate(self.handle, _items(specs), len(specs), ct, cp, C.byref(pol),
                                        C.c_void_p(phi_ptr), C.c_void_p(theta_ptr), reps)
        if st != ICP_OK and (raise_on_audit or st != ICP_ERR_AUDIT):
            check(st)
        return list(reps)

    def targets(self, phi_ptr: int, theta_ptr: int, count: int, target_ptr: int) -> None:
        check(LIB.icp_surrogate_targets(self.handle, C.c_void_p(phi_ptr), C.c_void_p(theta_ptr), count,
                                        C.c_void_p(target_ptr)))


# ------------------------------------------------------- Table-II rainbow diffraction
def rainbow_table_sigma(radius_mm: float) -> float:
    """Table-II primary width in degrees for a drop radius (mm, rounded to float32 first)."""
    out = C.c_double(0.0)
    check(LIB.icp_rainbow_table_sigma(float(np.float32(radius_mm)), C.byref(out)))
    return out.value


def diffraction_config(radius_mm: float, primary_sigma_deg: float = 0.0,
                       transition_contrast: float = 0.25) -> DiffractionConfig:
    """The diffraction settings PatchOptics derives from WaveOpticsSettings: a zero width
    selects Table II at the drop's radius (outside 0.1 .. 1.0 mm rejected), a positive one
    is an explicit extension; support 4 sigma, blend from 3 sigma."""
    sigma = float(primary_sigma_deg)
    if not (sigma >= 0.0 and math.isfinite(sigma)):
        raise InvalidArgument(ICP_ERR_INVALID_ARGUMENT, "Invalid diffraction sigma.")
    if sigma == 0.0:
        sigma = rainbow_table_sigma(radius_mm)
    return DiffractionConfig(sigma * math.pi / 180.0, 4.0, float(transition_contrast), 3.0)


@dataclass
class DiffractionOutput:
    transitions: np.ndarray  # uint32 [nt * np]: edge labels below each direction
    results: np.ndarray      # DIFFRACTION_DTYPE [nt * np]
    density: np.ndarray      # float64 [nt * np]: intensity_s + intensity_p (the stage's CDF input)
    stats: dict


def rainbow_diffraction(ctx: Context, focal, nt: int, np_: int, config: DiffractionConfig,
                        transitions=None) -> DiffractionOutput:
    """Table-II diffraction of a focal grid (FOCAL_DTYPE [nt * np], host or DeviceArray): the
    labels are detected unless given (uint32 [nt * np]), then every direction is filtered."""
    n = nt * np_
    if isinstance(focal, DeviceArray):
        df = focal
    else:
        df = DeviceArray(ctx, n, FOCAL_DTYPE).upload(np.ascontiguousarray(focal, dtype=FOCAL_DTYPE).reshape(-1))
    dt = DeviceArray(ctx, n, np.uint32)
    dr = DeviceArray(ctx, n, DIFFRACTION_DTYPE)
    dd = DeviceArray(ctx, n)
    stats = DiffractionStats()
    if transitions is None:
        check(LIB.icp_rainbow_diffraction(ctx.handle, df.ptr, nt, np_, C.byref(config), dt.ptr, dr.ptr, dd.ptr,
                                          C.byref(stats)))
    else:
        dt.upload(np.ascontiguousarray(transitions, dtype=np.uint32).reshape(-1))
        check(LIB.icp_rainbow_filter(ctx.handle, df.ptr, dt.ptr, nt, np_, C.byref(config), dr.ptr, dd.ptr,
                                     C.byref(stats)))
    return DiffractionOutput(dt.download(), dr.download(), dd.download(), stats.as_dict())


# ------------------------------------------------------------------ patch optics
@dataclass
class FoldedRecords:
    indices: np.ndarray    # uint32 [patch_count]: record of each compact patch, or 0xffffffff
    records: np.ndarray    # FOLDED_DTYPE [count], compact-index order
    stats: "FoldedStats"


def folded_prepare(ctx: Context, vertices: "DeviceArray", patches: "DeviceArray", patch_count: int, incident,
                   focal=None, config: "FoldedConfig | None" = None):
    """Folded-patch records of every NeedsRefinement patch (icp_folded_prepare) from device arrays:
    (device record indices, device records or None, count, FoldedStats)."""
    di = DeviceArray(ctx, max(1, patch_count), np.uint32)
    n = C.c_uint32(0)
    st = FoldedStats()
    k = (C.c_float * 3)(*map(float, incident))
    fc = None
    if focal is not None:
        w, h, e, q = focal
        fc = FocalConfig(w, h, e, 0, (C.c_uint32 * 4)(*q))
    cfg = C.byref(config) if config is not None else None
    args = (ctx.handle, vertices.ptr, vertices.count, patches.ptr, patch_count, k, C.byref(fc) if fc else None, cfg,
            di.ptr)
    rc = LIB.icp_folded_prepare(*args, None, 0, C.byref(n), C.byref(st))
    if n.value == 0:
        check(rc)
        return di, None, 0, st
    dr = DeviceArray(ctx, n.value, FOLDED_DTYPE)
    check(LIB.icp_folded_prepare(*args, dr.ptr, n.value, C.byref(n), C.byref(st)))
    return di, dr, n.value, st


def patch_optics(ctx: Context, vertices, patches, directions, offsets, summaries, hits, incident, incident_basis,
                 second=None, polarization: int | None = None, focal=None, folded: bool = False):
    """Per-direction optics of the drop's wave stages from host arrays (VERTEX_DTYPE, PATCH_DTYPE,
    float32 [n, 3] directions, uint64 [n + 1] hit offsets, SUMMARY_DTYPE [n], HIT_DTYPE, optional
    float32 [vertices, 4] second response column): the OPTICAL_DTYPE results and, with
    focal = (grid_width, grid_height, grid_half_extent, quarter_turn_offsets[4]), the focal stage
    (FOCAL_DTYPE, the input of rainbow_diffraction).  polarization defaults to unpolarized
    exactly when a second column is given.  With folded=True the NeedsRefinement patches get
    folded-patch records first (icp_folded_prepare) and the optics take them
    (icp_patch_optics_folded); the records come back as a third value (FoldedRecords)."""
    n = len(directions)
    arrays = [DeviceArray(ctx, len(a), dt).upload(np.ascontiguousarray(a, dtype=dt).reshape(-1))
              for a, dt in ((vertices, VERTEX_DTYPE), (patches, PATCH_DTYPE), (summaries, SUMMARY_DTYPE),
                            (hits, HIT_DTYPE))]
    dv, dp, ds, dh = arrays
    dd = DeviceArray(ctx, 3 * n, np.float32).upload(np.asarray(directions, dtype=np.float32).reshape(-1))
    do = DeviceArray(ctx, n + 1, np.uint64).upload(np.asarray(offsets, dtype=np.uint64))
    d2 = None
    if second is not None:
        d2 = DeviceArray(ctx, 4 * len(second), np.float32).upload(np.asarray(second, dtype=np.float32).reshape(-1))
    pol = (1 if second is not None else 0) if polarization is None else int(polarization)
    inp = OpticsInput(dv.ptr, dp.ptr, dd.ptr, do.ptr, ds.ptr, dh.ptr, d2.ptr if d2 else None, len(hits),
                      len(vertices), len(patches), n, 0 if second is None else len(second),
                      Vec3f(*map(float, incident)), Vec3f(*map(float, incident_basis)), pol, 0)
    dr = DeviceArray(ctx, n, OPTICAL_DTYPE)
    df = DeviceArray(ctx, n, FOCAL_DTYPE) if focal is not None else None
    fc = None
    if focal is not None:
        w, h, e, q = focal
        fc = FocalConfig(w, h, e, 0, (C.c_uint32 * 4)(*q))
    if not folded:
        check(LIB.icp_patch_optics(ctx.handle, C.byref(inp), dr.ptr, C.byref(fc) if fc is not None else None,
                                   df.ptr if df is not None else None))
        return dr.download(), (df.download() if df is not None else None)
    di, drec, count, st = folded_prepare(ctx, dv, dp, len(patches), incident, focal)
    view = FoldedView(di.ptr, drec.ptr if drec is not None else None, len(patches), count)
    check(LIB.icp_patch_optics_folded(ctx.handle, C.byref(inp), dr.ptr, C.byref(fc) if fc is not None else None,
                                      df.ptr if df is not None else None, C.byref(view) if drec is not None else None))
    recs = FoldedRecords(di.download()[:len(patches)], drec.download() if drec is not None else
                         np.zeros(0, FOLDED_DTYPE), st)
    return dr.download(), (df.download() if df is not None else None), recs


@dataclass
class PatchBuild:
    patches: np.ndarray    # PATCH_DTYPE [count], patch_id order
    aabbs: np.ndarray      # AABB_DTYPE [count]
    statuses: np.ndarray   # uint32 [4 (W-1)(H-1)], per cell
    histogram: list        # cells per status 0..7


def patch_build(ctx: Context, vertices, grid_width: int, grid_height: int, grid_half_extent: float) -> PatchBuild:
    """Patches of a four-family lattice (VERTEX_DTYPE [4 W H], host or DeviceArray)."""
    cells = 4 * (grid_width - 1) * (grid_height - 1)
    if isinstance(vertices, DeviceArray):
        dv = vertices
    else:
        dv = DeviceArray(ctx, len(vertices), VERTEX_DTYPE).upload(np.ascontiguousarray(vertices, dtype=VERTEX_DTYPE))
    dp = DeviceArray(ctx, cells, PATCH_DTYPE)
    db = DeviceArray(ctx, cells, AABB_DTYPE)
    ds = DeviceArray(ctx, cells, np.uint32)
    count = C.c_uint32(0)
    hist = (C.c_uint64 * 8)()
    check(LIB.icp_patch_build(ctx.handle, dv.ptr, grid_width, grid_height, float(grid_half_extent), dp.ptr, db.ptr,
                              ds.ptr, C.byref(count), hist))
    n = count.value
    return PatchBuild(dp.download()[:n], db.download()[:n], ds.download(), list(hist))


def raindrop_config(radius_mm: float, wavelength_nm: float, interior_index: float, incident_direction, grid: int,
                    sphere: bool = False, coefficients=None, grid_height: int | None = None) -> RaindropConfig:
    """RaindropSettings::make_config of an unpolarised trace (icp_raindrop_config_make)."""
    cfg = RaindropConfig()
    d = (C.c_float * 3)(*map(float, incident_direction))
    coef = None if coefficients is None else (C.c_float * 8)(*[float(x) for x in list(coefficients) + [0.0] * 8][:8])
    check(LIB.icp_raindrop_config_make(C.c_float(radius_mm), int(bool(sphere)), coef, C.c_float(wavelength_nm),
                                       C.c_float(interior_index), d, grid, grid if grid_height is None else grid_height,
                                       C.byref(cfg)))
    return cfg


@dataclass
class Lattice:
    vertices: "DeviceArray"      # VERTEX_DTYPE [4 W H], family-major
    second: "DeviceArray | None"  # float32 [4 W H, 4], the second response column
    stats: LatticeStats
    config: RaindropConfig


def lattice_trace(ctx: Context, config: RaindropConfig, unpolarized: bool = True) -> Lattice:
    """The four-family outgoing-ray lattice of one drop on the device (icp_lattice_trace)."""
    n = 4 * config.grid_width * config.grid_height
    dv = DeviceArray(ctx, n, VERTEX_DTYPE)
    ds = DeviceArray(ctx, n * 4, np.float32) if unpolarized else None
    st = LatticeStats()
    check(LIB.icp_lattice_trace(ctx.handle, C.byref(config), dv.ptr, ds.ptr if ds is not None else None,
                                C.byref(st)))
    return Lattice(dv, ds, st, config)


def query_directions(theta_count: int, phi_count: int, axis, e0) -> np.ndarray:
    """The reference's query grid directions, float32 [theta_count * phi_count, 3]."""
    out = np.empty((theta_count * phi_count, 3), dtype=np.float32)
    a = (C.c_float * 3)(*map(float, axis))
    b = (C.c_float * 3)(*map(float, e0))
    check(LIB.icp_query_directions(theta_count, phi_count, a, b, out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


@dataclass
class PatchQueryResult:
    offsets: np.ndarray    # uint64 [n + 1]
    summaries: np.ndarray  # SUMMARY_DTYPE [n]
    hits: np.ndarray       # HIT_DTYPE [offsets[n]]


def patch_query(ctx: Context, vertices, patches, aabbs, directions) -> PatchQueryResult:
    """All-hit query of patches (PATCH_DTYPE, AABB_DTYPE from patch_build) for float32 [n, 3]
    directions: sized first, then filled, as the reference's two query passes."""
    n = len(directions)
    dv = DeviceArray(ctx, len(vertices), VERTEX_DTYPE).upload(np.ascontiguousarray(vertices, dtype=VERTEX_DTYPE))
    dp = DeviceArray(ctx, max(1, len(patches)), PATCH_DTYPE)
    db = DeviceArray(ctx, max(1, len(aabbs)), AABB_DTYPE)
    if len(patches):
        dp.upload(np.ascontiguousarray(patches, dtype=PATCH_DTYPE))
        db.upload(np.ascontiguousarray(aabbs, dtype=AABB_DTYPE))
    dd = DeviceArray(ctx, max(1, 3 * n), np.float32)
    if n:
        dd.upload(np.asarray(directions, dtype=np.float32).reshape(-1))
    do = DeviceArray(ctx, n + 1, np.uint64)
    total = C.c_uint64(0)
    args = (ctx.handle, dv.ptr, len(vertices), dp.ptr, db.ptr, len(patches), dd.ptr, n, do.ptr)
    check(LIB.icp_patch_query(*args, None, None, 0, C.byref(total)))
    ds = DeviceArray(ctx, max(1, n), SUMMARY_DTYPE)
    dh = DeviceArray(ctx, max(1, total.value), HIT_DTYPE)
    check(LIB.icp_patch_query(*args, ds.ptr, dh.ptr, max(1, total.value), C.byref(total)))
    return PatchQueryResult(do.download(), ds.download()[:n], dh.download()[:total.value])


# ----------------------------------------------------------- wave-stage CDF input
def _device(ctx: Context, a, dtype):
    if a is None or isinstance(a, DeviceArray):
        return a
    a = np.ascontiguousarray(a, dtype=dtype).reshape(-1)
    return DeviceArray(ctx, len(a), dtype).upload(a)


def stage_density(ctx: Context, stage: str, optical, focal=None, diffraction=None) -> tuple[DeviceArray, dict]:
    """The density of a wave stage per query direction (device) and the CDF builder's input
    audit (maximum, invalid values, incomplete and underresolved directions, first problem)."""
    do = _device(ctx, optical, OPTICAL_DTYPE)
    df = _device(ctx, focal, FOCAL_DTYPE)
    dr = _device(ctx, diffraction, DIFFRACTION_DTYPE)
    dd = DeviceArray(ctx, do.count)
    rep = DensityReport()
    check(LIB.icp_stage_density(ctx.handle, WAVE_STAGES[stage], do.ptr, df.ptr if df else None, dr.ptr if dr else None,
                                do.count, dd.ptr, C.byref(rep)))
    return dd, rep.as_dict()


def density_gate(report: dict, allow_underresolved: bool = False) -> None:
    """The reference's CDF input gate: raises AuditError on an invalid value, an incomplete
    direction, no positive density, or (unless allowed) an underresolved direction."""
    if (report["invalid_values"] or report["incomplete"] or not report["maximum"] > 0
            or (not allow_underresolved and report["underresolved"])):
        raise AuditError(ICP_ERR_AUDIT, "CDF input rejected: max_intensity={maximum}, invalid_values={invalid_values}, "
                                        "incomplete={incomplete}, underresolved={underresolved}".format(**report))


def stage_record(ctx: Context, stage: str, nt: int, np_: int, optical, focal=None, diffraction=None,
                 ct: int | None = None, cp: int | None = None, allow_underresolved: bool = False,
                 **policy) -> CdfResult:
    """A record of one wave stage from its per-direction results on the nt x np query grid:
    density, input gate, then the stored CDF (PhaseCdf.build with density input)."""
    dd, rep = stage_density(ctx, stage, optical, focal, diffraction)
    density_gate(rep, allow_underresolved)
    return PhaseCdf(ctx).build(dd, nt, np_, ct, cp, density=True, **policy)
