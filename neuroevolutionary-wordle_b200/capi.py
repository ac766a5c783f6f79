"""ctypes bindings of the runtime's C ABI (include/nwg_capi.h).

The product is the CUDA library libnwg.so built in this directory; this module only binds it.
There is no fallback: loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
from functools import lru_cache
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libnwg.so"
CATALOG_CAPACITY = 4739
_sz = C.c_size_t
_vp = C.c_void_p


class NwgError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where}: status {status} ({status_string(status)})")
        self.status = status


class RuntimeConfig(C.Structure):
    _fields_ = [(n, _sz) for n in ("genotype_slab_byte_budget_bytes", "generation_byte_budget_bytes",
                                   "host_spillover_byte_budget_bytes", "action_count", "population_size_ceiling",
                                   "grid_column_count")]


class WordCountSchedule(C.Structure):
    _fields_ = [("initial_word_count", _sz), ("word_count_step", _sz), ("word_count_step_period_generations", _sz)]


class RuntimeWordCounts(C.Structure):
    _fields_ = [("training_word_count", _sz), ("action_space_word_count", _sz),
                ("training_word_schedule", WordCountSchedule), ("shard_initial_radius", _sz),
                ("shard_radius_growth_period_generations", _sz)]


class ShardReleaseHistory(C.Structure):
    _fields_ = [("release_generations", _sz * CATALOG_CAPACITY), ("release_fitness_p99", C.c_float * CATALOG_CAPACITY),
                ("release_count", _sz)]


class FitnessSummary(C.Structure):
    _fields_ = [("best_fitness", C.c_float), ("average_fitness", C.c_float), ("best_index", _sz),
                ("best_slot_index", C.c_uint32), ("generation_index", _sz), ("action_count", _sz),
                ("population_size", _sz)]


class ParentSelectionConfig(C.Structure):
    _fields_ = [("cellular_breeding_radius", _sz), ("rank_exponent", C.c_float)]


class BreedingConfig(C.Structure):
    _fields_ = [("crossover_temperature_level1", C.c_float), ("crossover_temperature_level2", C.c_float),
                ("crossover_temperature_level3", C.c_float)]


class MutationConfig(C.Structure):
    _fields_ = [("mutation_probability", C.c_float), ("mutation_sigma", C.c_float),
                ("output_tail_row_scale_mutation_probability", C.c_float)]


class AssemblyConfig(C.Structure):
    _fields_ = [("parent_selection", ParentSelectionConfig), ("breeding", BreedingConfig),
                ("mutation", MutationConfig)]


class PendingInjection(C.Structure):
    _fields_ = [("enabled", C.c_bool), ("first_catalog_word_index", _sz), ("injection_count", _sz)]


class EvaluationStats(C.Structure):
    _fields_ = [("game_steps", C.c_uint64), ("episodes", C.c_uint64), ("encoded_turns", C.c_uint64),
                ("fitness_mean_fp64", C.c_double), ("fitness_variance_fp64", C.c_double),
                ("eval_kernel_ms", C.c_double), ("rescored_chunks", C.c_uint64), ("full_rescores", C.c_uint64),
                ("candidate_chunks", C.c_uint64), ("fallback_steps", C.c_uint64)]


FORM_FP32, FORM_TC_BF16, FORM_TC_FP16, FORM_TC_TRUNK_BF16, FORM_TC_TRUNK_FP16 = 0, 1, 2, 3, 4


class RuntimeInfo(C.Structure):
    _fields_ = [(n, _sz) for n in ("action_count", "slot_stride_bytes", "slot_pitch_bytes", "slot_count",
                                   "max_generation_size", "grid_column_count", "current_generation_index",
                                   "current_generation_size", "next_generation_index", "next_generation_size",
                                   "planned_child_count", "slab_bytes", "generation_byte_budget_bytes",
                                   "host_spillover_byte_budget_bytes", "epicenter_row_count")] + [
        ("prepared", C.c_uint32)]


class SlabLayout(C.Structure):
    _fields_ = [(n, _sz) for n in ("action_count", "slot_stride_bytes", "slot_count", "slab_bytes")]


class GridShape(C.Structure):
    _fields_ = [(n, _sz) for n in ("row_count", "column_count", "cell_count")]


class GraphInfo(C.Structure):
    _fields_ = [(n, _sz) for n in ("launches", "instantiations", "updates")]


class LaunchTuning(C.Structure):
    _fields_ = [("decided", C.c_int), ("trials", C.c_int), ("eval_ctas", C.c_int), ("breed_warps", C.c_int),
                ("eval_ms", C.c_float * 2), ("breed_ms", C.c_float * 3)]


class CheckpointRecord(C.Structure):
    """nwg_checkpoint: RuntimeCheckpoint (slab_runtime.hpp:86-117) with its vectors as pointers."""
    _fields_ = [("schema_version", C.c_uint32), ("genome_layout_version", C.c_uint32), ("resume_phase", C.c_uint32),
                ("checksum", C.c_uint64), ("training_data_identity_hash", C.c_uint64),
                ("generation_seed", C.c_uint32), ("runtime_word_counts", RuntimeWordCounts),
                ("training_shard_release_history", ShardReleaseHistory), ("assembly_config", AssemblyConfig),
                ("pending_output_embedding_injection", PendingInjection), ("runtime_config", RuntimeConfig),
                ("slab_layout", SlabLayout), ("current_grid_shape", GridShape), ("next_grid_shape", GridShape),
                ("epicenter_grid_shape", GridShape), ("generation_index", _sz), ("individual_count", _sz),
                ("slot_indices", _vp), ("fitness", _vp), ("evaluation_counts", _vp), ("has_fitness", _vp),
                ("child_count", _sz), ("parent_pairs", _vp), ("live_count", _sz), ("live_organisms", _vp),
                ("live_genomes", _vp)]


class WinnerMetadata(C.Structure):
    """nwg_winner_metadata: WinnerArtifactMetadata (model_artifact/winner_artifact.hpp:12-21) minus its path."""
    _fields_ = [("best_fitness", C.c_float), ("generation_index", _sz), ("best_index", _sz),
                ("best_slot_index", C.c_uint32), ("action_count", _sz), ("genome_byte_count", _sz),
                ("seed", C.c_uint32)]


class FitnessTelemetry(C.Structure):
    """nwg_fitness_telemetry: GenerationFitnessTelemetryRow (cli/run_genetic_algorithm.cu:594-610)."""
    _fields_ = [("generation", _sz), ("population_size", _sz), ("training_word_count", _sz)] + [
        (n, C.c_float) for n in ("fitness_min", "fitness_mean", "fitness_median", "fitness_p90", "fitness_p99",
                                 "fitness_max", "fitness_stddev")] + [
        ("distinct_fitness_count", _sz), ("has_breeding_metrics", C.c_bool), ("parent_childless_count", _sz),
        ("parent_one_child_count", _sz), ("parent_multiple_children_count", _sz)]


class ConvergenceTelemetry(C.Structure):
    """nwg_convergence_telemetry: GeneticConvergenceTelemetryRow (cli/run_genetic_algorithm.cu:612-624)."""
    _fields_ = [(n, _sz) for n in ("generation", "sample_organisms", "sample_weights", "pair_count")] + [
        (n, C.c_float) for n in ("centroid_distance_mean", "centroid_distance_min", "centroid_distance_max",
                                 "pairwise_distance_mean", "pairwise_distance_min", "pairwise_distance_max",
                                 "elapsed_ms")]


class ShardReleasePolicy(C.Structure):
    """nwg_shard_release_policy; defaults of training_folder/training_data.hpp:17-20."""
    _fields_ = [("min_gap_generations", _sz), ("first_new_release_generation", _sz),
                ("centroid_distance_threshold", C.c_float), ("fitness_p99_threshold", C.c_float)]

    def __init__(self, min_gap_generations=3, first_new_release_generation=10, centroid_distance_threshold=6.0,
                 fitness_p99_threshold=0.20):
        super().__init__(min_gap_generations, first_new_release_generation, centroid_distance_threshold,
                         fitness_p99_threshold)


class SelectedAction(C.Structure):
    """nwg_selected_action: SelectedAction (model/output_embedding/output_embedding.hpp:35-39)."""
    _fields_ = [("word", C.c_uint8 * 5), ("score", C.c_float), ("action_index", _sz)]


class SurrogateConfig(C.Structure):
    """nwg_surrogate_config (defaults of the learned-surrogate method)."""
    _fields_ = [("candidates_per_cell", _sz), ("audit_fraction", C.c_float), ("spearman_floor", C.c_float),
                ("replay_capacity", _sz), ("warmup_pairs", _sz), ("train_steps", _sz), ("batch_rows", _sz),
                ("learning_rate", C.c_float), ("seed", C.c_uint32), ("evaluation_form", C.c_int),
                ("margin_tau", C.c_float)]

    def __init__(self, candidates_per_cell=4, audit_fraction=0.05, spearman_floor=0.6, replay_capacity=65536,
                 warmup_pairs=8192, train_steps=8, batch_rows=1024, learning_rate=1e-4, seed=0, evaluation_form=4,
                 margin_tau=1e-3):
        super().__init__(candidates_per_cell, audit_fraction, spearman_floor, replay_capacity, warmup_pairs,
                         train_steps, batch_rows, learning_rate, seed, evaluation_form, margin_tau)


class SurrogateStats(C.Structure):
    _fields_ = [("generation", _sz), ("candidates", _sz), ("evaluated", _sz), ("screened", C.c_bool),
                ("spearman", C.c_float), ("train_loss", C.c_float), ("train_steps", _sz), ("replay_size", _sz),
                ("mean_fitness", C.c_double), ("mean_solve_rate", C.c_double), ("mean_fitness_model_pick", C.c_double),
                ("mean_fitness_first_candidate", C.c_double), ("mean_fitness_best_candidate", C.c_double),
                ("game_steps", C.c_uint64)] + [
        (n, C.c_float) for n in ("ms_select_breed", "ms_descriptors", "ms_inference", "ms_evaluation", "ms_training",
                                 "ms_install", "ms_total")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


POST_FITNESS_FN = C.CFUNCTYPE(C.c_bool, _vp, C.POINTER(RuntimeWordCounts), _vp)
SHARD_RELEASE_FN = C.CFUNCTYPE(C.c_bool, _vp, C.POINTER(RuntimeWordCounts), C.POINTER(PendingInjection), _vp)

EXPORTS = [
    "nwg_abi_version", "nwg_status_string", "nwg_upload_catalog", "nwg_create", "nwg_destroy", "nwg_set_stream",
    "nwg_get_info", "nwg_set_evaluation_form", "nwg_set_margin_guard", "nwg_bootstrap", "nwg_set_cell_words", "nwg_evaluate", "nwg_read_summary",
    "nwg_read_evaluation_stats", "nwg_advance", "nwg_advance_graphed", "nwg_hint_groups_available", "nwg_read_graph_info",
    "nwg_read_launch_tuning", "nwg_set_launch_tuning", "nwg_swap_generations", "nwg_read_status",
    "nwg_download_current_generation", "nwg_download_slot", "nwg_upload_slot", "nwg_upload_current_generation",
    "nwg_download_assembly_plan", "nwg_device_slab", "nwg_evaluate_traced", "nwg_select_parents_device",
    "nwg_breed_device", "nwg_bootstrap_device", "nwg_evaluate_noalloc", "nwg_prepare_generation",
    "nwg_assemble_prepared", "nwg_checkpoint_capture", "nwg_checkpoint_restore", "nwg_checkpoint_resume",
    "nwg_checkpoint_write", "nwg_checkpoint_read", "nwg_checkpoint_free", "nwg_checkpoint_checksum",
    "nwg_checkpoint_identity_hash", "nwg_winner_artifact_write", "nwg_winner_artifact_persist",
    "nwg_winner_artifact_read", "nwg_download_next_generation", "nwg_fitness_telemetry_collect",
    "nwg_convergence_telemetry_collect", "nwg_convergence_sample_plan", "nwg_maybe_release_training_shard",
    "nwg_single_model_create", "nwg_single_model_destroy", "nwg_single_model_set_stream", "nwg_single_model_select",
    "nwg_read_solve_rates", "nwg_read_score_table", "nwg_mlp_create", "nwg_mlp_destroy", "nwg_mlp_set_stream", "nwg_mlp_parameter_count",
    "nwg_mlp_parameters", "nwg_mlp_forward", "nwg_mlp_gradients", "nwg_mlp_train_step", "nwg_bf16_gemm_nt",
    "nwg_descriptors", "nwg_surrogate_create", "nwg_surrogate_destroy", "nwg_surrogate_advance",
    "nwg_set_band", "nwg_device_generation", "nwg_band_prepare", "nwg_band_copy_rows", "nwg_band_install_halo",
    "nwg_measure_fp32_peak", "nwg_set_wait_limit",
]


@lru_cache(None)
def lib() -> C.CDLL:
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} is not built; run neuroevolutionary-wordle_b200/build.py")
    L = C.CDLL(str(LIB_PATH))
    L.nwg_status_string.restype = C.c_char_p
    L.nwg_status_string.argtypes = [C.c_int]
    L.nwg_upload_catalog.argtypes = [_vp, _sz]
    L.nwg_create.argtypes = [C.POINTER(RuntimeConfig), C.POINTER(_vp)]
    L.nwg_destroy.argtypes = [_vp]
    L.nwg_destroy.restype = None
    L.nwg_set_stream.argtypes = [_vp, _vp]
    L.nwg_get_info.argtypes = [_vp, C.POINTER(RuntimeInfo)]
    L.nwg_bootstrap.argtypes = [_vp, _sz, C.c_uint32, _sz]
    L.nwg_set_evaluation_form.argtypes = [_vp, C.c_int]
    L.nwg_set_margin_guard.argtypes = [_vp, C.c_float]
    L.nwg_set_cell_words.argtypes = [_vp, _vp, _vp, _sz]
    L.nwg_evaluate.argtypes = [_vp, C.POINTER(RuntimeWordCounts), C.POINTER(ShardReleaseHistory)]
    L.nwg_read_summary.argtypes = [_vp, C.POINTER(FitnessSummary)]
    L.nwg_read_evaluation_stats.argtypes = [_vp, C.POINTER(EvaluationStats)]
    L.nwg_advance.argtypes = [_vp, C.c_uint32, C.POINTER(RuntimeWordCounts), C.POINTER(AssemblyConfig),
                              C.POINTER(PendingInjection), POST_FITNESS_FN, _vp, SHARD_RELEASE_FN, _vp,
                              C.POINTER(ShardReleaseHistory)]
    L.nwg_prepare_generation.argtypes = L.nwg_advance.argtypes
    L.nwg_advance_graphed.argtypes = [_vp, C.c_uint32, C.POINTER(RuntimeWordCounts), C.POINTER(AssemblyConfig),
                                      C.POINTER(PendingInjection)]
    L.nwg_read_graph_info.argtypes = [_vp, C.POINTER(GraphInfo)]
    L.nwg_hint_groups_available.argtypes = [_vp, _sz, _vp]
    L.nwg_read_launch_tuning.argtypes = [_vp, _sz, C.c_int, C.POINTER(LaunchTuning)]
    L.nwg_set_launch_tuning.argtypes = [_vp, C.c_int]
    L.nwg_assemble_prepared.argtypes = [_vp]
    L.nwg_checkpoint_capture.argtypes = L.nwg_advance.argtypes + [_vp, _sz, C.POINTER(CheckpointRecord)]
    L.nwg_checkpoint_restore.argtypes = [C.POINTER(CheckpointRecord), C.POINTER(_vp)]
    L.nwg_checkpoint_resume.argtypes = [_vp]
    L.nwg_checkpoint_write.argtypes = [C.POINTER(CheckpointRecord), C.c_char_p]
    L.nwg_checkpoint_read.argtypes = [C.c_char_p, C.POINTER(CheckpointRecord)]
    L.nwg_checkpoint_free.argtypes = [C.POINTER(CheckpointRecord)]
    L.nwg_checkpoint_free.restype = None
    L.nwg_checkpoint_checksum.argtypes = [C.POINTER(CheckpointRecord)]
    L.nwg_checkpoint_checksum.restype = C.c_uint64
    L.nwg_checkpoint_identity_hash.argtypes = [C.POINTER(RuntimeWordCounts), C.POINTER(ShardReleaseHistory), _vp,
                                               _sz]
    L.nwg_checkpoint_identity_hash.restype = C.c_uint64
    L.nwg_winner_artifact_write.argtypes = [C.c_char_p, C.c_char_p, _vp, C.POINTER(WinnerMetadata), _vp, _sz,
                                            C.c_char_p, C.c_char_p]
    L.nwg_winner_artifact_persist.argtypes = [_vp, C.c_uint32, _vp, _sz, C.c_char_p, C.c_char_p, C.c_char_p,
                                              C.c_char_p]
    L.nwg_winner_artifact_read.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(WinnerMetadata), _vp, _sz, _vp,
                                           C.POINTER(_sz), C.c_char_p, _sz, C.c_char_p, _sz]
    L.nwg_fitness_telemetry_collect.argtypes = [_vp, C.POINTER(RuntimeWordCounts), C.c_bool,
                                                C.POINTER(FitnessTelemetry)]
    L.nwg_convergence_telemetry_collect.argtypes = [_vp, C.c_uint32, C.POINTER(ConvergenceTelemetry)]
    L.nwg_convergence_sample_plan.argtypes = [_sz, _sz, C.c_uint32, _sz, _vp, C.POINTER(_sz), _vp, C.POINTER(_sz),
                                              _vp, C.POINTER(_sz)]
    L.nwg_maybe_release_training_shard.argtypes = [_vp, C.POINTER(RuntimeWordCounts), C.POINTER(ShardReleasePolicy),
                                                   _sz, C.c_uint32, C.POINTER(ShardReleaseHistory),
                                                   C.POINTER(PendingInjection), C.POINTER(_sz),
                                                   C.POINTER(FitnessTelemetry), C.POINTER(ConvergenceTelemetry)]
    L.nwg_single_model_create.argtypes = [_vp, _sz, _vp, _sz, C.POINTER(_vp)]
    L.nwg_single_model_destroy.argtypes = [_vp]
    L.nwg_single_model_destroy.restype = None
    L.nwg_single_model_set_stream.argtypes = [_vp, _vp]
    L.nwg_single_model_select.argtypes = [_vp, _vp, _vp, _vp, _sz, C.POINTER(SelectedAction)]
    L.nwg_read_solve_rates.argtypes = [_vp, _vp, _sz, C.POINTER(_sz), C.POINTER(C.c_double)]
    L.nwg_read_score_table.argtypes = [_vp, _sz, _vp, _sz, C.POINTER(_sz)]
    L.nwg_mlp_create.argtypes = [_sz, C.c_uint32, C.c_float, C.POINTER(_vp)]
    L.nwg_mlp_destroy.argtypes = [_vp]
    L.nwg_mlp_destroy.restype = None
    L.nwg_mlp_set_stream.argtypes = [_vp, _vp]
    L.nwg_mlp_parameter_count.restype = _sz
    L.nwg_mlp_parameters.argtypes = [_vp, _vp, _vp]
    L.nwg_mlp_forward.argtypes = [_vp, _vp, _sz, _vp]
    L.nwg_mlp_gradients.argtypes = [_vp, _vp, _vp, _sz, _vp, C.POINTER(C.c_float)]
    L.nwg_mlp_train_step.argtypes = [_vp, _vp, _vp, _sz]
    L.nwg_bf16_gemm_nt.argtypes = [_vp, _sz, _vp, _sz, _vp, _sz, _sz, _sz, _sz, _vp]
    L.nwg_descriptors.argtypes = [_vp, _sz, _vp, _sz, _vp, _vp, _vp, C.c_float, _vp, _vp]
    L.nwg_surrogate_create.argtypes = [_vp, C.POINTER(SurrogateConfig), _vp, _sz, _vp, _sz, C.POINTER(_vp)]
    L.nwg_surrogate_destroy.argtypes = [_vp]
    L.nwg_surrogate_destroy.restype = None
    L.nwg_surrogate_advance.argtypes = [_vp, C.c_uint32, C.POINTER(RuntimeWordCounts), C.POINTER(AssemblyConfig),
                                        C.POINTER(SurrogateStats)]
    L.nwg_swap_generations.argtypes = [_vp]
    L.nwg_read_status.argtypes = [_vp, C.POINTER(C.c_int)]
    L.nwg_download_current_generation.argtypes = [_vp, _vp, _vp, _vp, _vp, _sz, C.POINTER(_sz), C.POINTER(_sz)]
    L.nwg_download_slot.argtypes = [_vp, C.c_uint32, _vp, _sz, C.POINTER(_sz)]
    L.nwg_upload_slot.argtypes = [_vp, C.c_uint32, _vp, _sz]
    L.nwg_upload_current_generation.argtypes = [_vp, _vp, _sz, _sz]
    L.nwg_download_assembly_plan.argtypes = [_vp, _vp, _sz, C.POINTER(_sz)]
    L.nwg_device_slab.argtypes = [_vp, C.POINTER(_vp), C.POINTER(_sz)]
    L.nwg_evaluate_traced.argtypes = [_vp, C.POINTER(RuntimeWordCounts), C.POINTER(ShardReleaseHistory), _sz, _vp,
                                      _vp, _vp, _vp]
    L.nwg_select_parents_device.argtypes = [_vp, _vp, _sz, _sz, _sz, _sz, C.POINTER(ParentSelectionConfig),
                                            C.c_uint32, _vp, _vp]
    L.nwg_breed_device.argtypes = [_vp, _sz, _vp, _vp, _sz, _vp, _sz, _sz, C.c_uint32, _sz,
                                   C.POINTER(BreedingConfig), C.POINTER(MutationConfig), _vp]
    L.nwg_bootstrap_device.argtypes = [_vp, _sz, _sz, _sz, C.c_uint32, _sz, _vp]
    L.nwg_set_band.argtypes = [_vp, _sz, _sz, _sz]
    L.nwg_device_generation.argtypes = [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_sz)]
    L.nwg_band_prepare.argtypes = [_vp, C.c_uint32, C.POINTER(AssemblyConfig), _vp, _vp]
    L.nwg_band_copy_rows.argtypes = [_vp, _sz, _sz, _vp, _sz]
    L.nwg_band_install_halo.argtypes = [_vp, _vp, _vp, _sz]
    L.nwg_measure_fp32_peak.argtypes = [C.POINTER(C.c_double), _vp]
    L.nwg_set_wait_limit.argtypes = [_vp, C.c_uint32]
    return L


def measure_fp32_peak(stream: int | None = None) -> float:
    """FP32 FMA throughput of the current device (TFLOP/s), measured by the library's peak kernel."""
    v = C.c_double()
    check(lib().nwg_measure_fp32_peak(C.byref(v), stream), "nwg_measure_fp32_peak")
    return v.value


def status_string(status: int) -> str:
    return lib().nwg_status_string(status).decode()


def check(status: int, where: str) -> None:
    if status != 0:
        raise NwgError(status, where)


def _np_ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def hint_groups_available(letters: np.ndarray) -> np.ndarray:
    """Per word (rows of 5 letter indices): whether it has the hint-grid group an injection needs."""
    words = np.ascontiguousarray(letters, np.uint8).reshape(-1, 5)
    out = np.zeros(len(words), np.uint8)
    check(lib().nwg_hint_groups_available(_np_ptr(words), len(words), _np_ptr(out)), "nwg_hint_groups_available")
    return out.astype(bool)


def genome_stride_bytes(action_count: int) -> int:
    """Reference genome image size (genetic_algorithm/genome/dynamic_layout.hpp:30-36)."""
    return 0 if action_count == 0 else ((301056 + 76 * action_count + 1) // 2) * 2


def upload_catalog(letters: np.ndarray) -> None:
    letters = np.ascontiguousarray(letters, np.uint8).reshape(-1, 5)
    check(lib().nwg_upload_catalog(_np_ptr(letters), len(letters)), "nwg_upload_catalog")


def word_counts(training: int, action_space: int, initial: int | None = None, step: int = 0, period: int = 1,
                initial_radius: int = 0, growth_period: int = 2) -> RuntimeWordCounts:
    wc = RuntimeWordCounts()
    wc.training_word_count = training
    wc.action_space_word_count = action_space
    wc.training_word_schedule.initial_word_count = training if initial is None else initial
    wc.training_word_schedule.word_count_step = step
    wc.training_word_schedule.word_count_step_period_generations = period
    wc.shard_initial_radius = initial_radius
    wc.shard_radius_growth_period_generations = growth_period
    return wc


def assembly_config(radius=2, rank_exponent=0.5, l1=0.02, l2=0.01, l3=0.005, p=1e-4, sigma=0.02,
                    row_scale=0.0) -> AssemblyConfig:
    cfg = AssemblyConfig()
    cfg.parent_selection.cellular_breeding_radius = radius
    cfg.parent_selection.rank_exponent = rank_exponent
    cfg.breeding.crossover_temperature_level1 = l1
    cfg.breeding.crossover_temperature_level2 = l2
    cfg.breeding.crossover_temperature_level3 = l3
    cfg.mutation.mutation_probability = p
    cfg.mutation.mutation_sigma = sigma
    cfg.mutation.output_tail_row_scale_mutation_probability = row_scale
    return cfg


class Runtime:
    """One device GA runtime (DeviceSlabGARuntimeBuffers of the reference)."""

    def __init__(self, action_count: int, population: int, columns: int, slab_generations: float = 2.0,
                 stream: int | None = None, slab_slots: int | None = None):
        stride = genome_stride_bytes(action_count)
        cfg = RuntimeConfig()
        cfg.generation_byte_budget_bytes = population * stride
        slots = slab_slots if slab_slots is not None else int(slab_generations * population)
        cfg.genotype_slab_byte_budget_bytes = slots * stride
        cfg.host_spillover_byte_budget_bytes = 0
        cfg.action_count = action_count
        cfg.population_size_ceiling = population
        cfg.grid_column_count = columns
        handle = _vp()
        check(lib().nwg_create(C.byref(cfg), C.byref(handle)), "nwg_create")
        self.handle = handle
        self.action_count = action_count
        self.population = population
        self.columns = columns
        self._form = FORM_FP32
        self._keep = []
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if self.handle:
            lib().nwg_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream: int) -> None:
        check(lib().nwg_set_stream(self.handle, stream), "nwg_set_stream")

    def info(self) -> RuntimeInfo:
        info = RuntimeInfo()
        check(lib().nwg_get_info(self.handle, C.byref(info)), "nwg_get_info")
        return info

    def set_form(self, form: int) -> None:
        check(lib().nwg_set_evaluation_form(self.handle, form), "nwg_set_evaluation_form")
        self._form = form

    def set_margin_guard(self, tau: float) -> None:
        check(lib().nwg_set_margin_guard(self.handle, tau), "nwg_set_margin_guard")

    DEFAULT_WAIT_LIMIT = 1 << 26

    def set_wait_limit(self, polls: int) -> None:
        """Poll limit of the tensor-core kernels' bounded waits (NWG_TIMEOUT when one gives up)."""
        check(lib().nwg_set_wait_limit(self.handle, polls), "nwg_set_wait_limit")

    def bootstrap(self, size: int, seed: int, generation_index: int = 0) -> None:
        check(lib().nwg_bootstrap(self.handle, size, seed, generation_index), "nwg_bootstrap")

    def set_cell_words(self, offsets: np.ndarray | None, words: np.ndarray | None) -> None:
        if offsets is None:
            check(lib().nwg_set_cell_words(self.handle, None, None, 0), "nwg_set_cell_words")
            return
        offsets = np.ascontiguousarray(offsets, np.uint32)
        words = np.ascontiguousarray(words, np.uint32)
        check(lib().nwg_set_cell_words(self.handle, _np_ptr(offsets), _np_ptr(words), len(offsets) - 1),
              "nwg_set_cell_words")

    def evaluate(self, counts: RuntimeWordCounts, history: ShardReleaseHistory | None = None) -> None:
        check(lib().nwg_evaluate(self.handle, C.byref(counts), C.byref(history) if history else None),
              "nwg_evaluate")

    def evaluate_traced(self, counts, trace_episodes, choices=0, turns=0, scores=0, policy=0, history=None) -> None:
        check(lib().nwg_evaluate_traced(self.handle, C.byref(counts), C.byref(history) if history else None,
                                        trace_episodes, choices or None, turns or None, scores or None,
                                        policy or None), "nwg_evaluate_traced")

    def summary(self) -> FitnessSummary:
        s = FitnessSummary()
        check(lib().nwg_read_summary(self.handle, C.byref(s)), "nwg_read_summary")
        return s

    def stats(self) -> EvaluationStats:
        s = EvaluationStats()
        check(lib().nwg_read_evaluation_stats(self.handle, C.byref(s)), "nwg_read_evaluation_stats")
        return s

    @classmethod
    def _adopt(cls, handle: C.c_void_p) -> "Runtime":
        """Wraps a runtime made by the library (a restored checkpoint's)."""
        rt = cls.__new__(cls)
        rt.handle = handle
        rt._keep = []
        rt._form = FORM_FP32
        info = rt.info()
        rt.action_count = info.action_count
        rt.population = info.max_generation_size
        rt.columns = info.grid_column_count
        return rt

    def _boundary_args(self, seed, counts, config, pending, post_fitness, shard_release, history):
        pf = POST_FITNESS_FN(post_fitness) if post_fitness else POST_FITNESS_FN()
        sr = SHARD_RELEASE_FN(shard_release) if shard_release else SHARD_RELEASE_FN()
        self._callbacks = (pf, sr)
        return (self.handle, seed, C.byref(counts), C.byref(config) if config else None,
                C.byref(pending) if pending else None, pf, None, sr, None, C.byref(history) if history else None)

    def advance(self, seed: int, counts: RuntimeWordCounts, config: AssemblyConfig | None = None,
                pending: PendingInjection | None = None, post_fitness=None, shard_release=None,
                history: ShardReleaseHistory | None = None) -> None:
        check(lib().nwg_advance(*self._boundary_args(seed, counts, config, pending, post_fitness, shard_release,
                                                     history)), "nwg_advance")
        self.action_count = self.info().action_count  # an injection widens the action space

    def advance_graphed(self, seed: int, counts: RuntimeWordCounts, config: AssemblyConfig | None = None,
                        pending: PendingInjection | None = None) -> None:
        """One generation with its device work launched as a CUDA graph (launch shapes tuned per width)."""
        check(lib().nwg_advance_graphed(self.handle, seed, C.byref(counts), C.byref(config) if config else None,
                                        C.byref(pending) if pending else None), "nwg_advance_graphed")
        self.action_count = self.info().action_count

    def graph_info(self) -> GraphInfo:
        g = GraphInfo()
        check(lib().nwg_read_graph_info(self.handle, C.byref(g)), "nwg_read_graph_info")
        return g

    def launch_tuning(self, width: int | None = None, form: int | None = None) -> LaunchTuning:
        t = LaunchTuning()
        info = self.info()
        check(lib().nwg_read_launch_tuning(self.handle, info.action_count if width is None else width,
                                           self._form if form is None else form, C.byref(t)),
              "nwg_read_launch_tuning")
        return t

    def set_launch_tuning(self, enabled: bool) -> None:
        check(lib().nwg_set_launch_tuning(self.handle, 1 if enabled else 0), "nwg_set_launch_tuning")

    def prepare(self, seed: int, counts: RuntimeWordCounts, config: AssemblyConfig | None = None,
                pending: PendingInjection | None = None, post_fitness=None, shard_release=None,
                history: ShardReleaseHistory | None = None) -> None:
        """The first half of advance: evaluate, run the callbacks, plan the next generation's parents."""
        check(lib().nwg_prepare_generation(*self._boundary_args(seed, counts, config, pending, post_fitness,
                                                                shard_release, history)), "nwg_prepare_generation")

    def persist_winner(self, binary_path, metadata_path, seed: int, catalog: np.ndarray, action_space_path="",
                       timestamp: str | None = None) -> None:
        """TryPersistWinningGenome: the last evaluation's best individual as a winner artefact."""
        cat = np.ascontiguousarray(catalog, np.uint8)
        check(lib().nwg_winner_artifact_persist(self.handle, seed, _np_ptr(cat), len(cat), str(action_space_path).encode(),
                                                str(binary_path).encode(), str(metadata_path).encode(),
                                                timestamp.encode() if timestamp is not None else None),
              "nwg_winner_artifact_persist")

    def fitness_telemetry(self, counts: RuntimeWordCounts | None = None, with_breeding: bool = False):
        row = FitnessTelemetry()
        check(lib().nwg_fitness_telemetry_collect(self.handle, C.byref(counts) if counts else None, with_breeding,
                                                  C.byref(row)), "nwg_fitness_telemetry_collect")
        return row

    def convergence_telemetry(self, run_seed: int):
        row = ConvergenceTelemetry()
        check(lib().nwg_convergence_telemetry_collect(self.handle, run_seed, C.byref(row)),
              "nwg_convergence_telemetry_collect")
        return row

    def maybe_release_training_shard(self, counts: RuntimeWordCounts, policy: ShardReleasePolicy,
                                     catalog_word_count: int, run_seed: int, history: ShardReleaseHistory):
        """TryMaybeReleaseTrainingDataShard: (pending injection, next word count, fitness row, convergence row)."""
        pending = PendingInjection()
        nxt = _sz()
        f = FitnessTelemetry()
        c = ConvergenceTelemetry()
        check(lib().nwg_maybe_release_training_shard(self.handle, C.byref(counts), C.byref(policy),
                                                     catalog_word_count, run_seed, C.byref(history), C.byref(pending),
                                                     C.byref(nxt), C.byref(f), C.byref(c)),
              "nwg_maybe_release_training_shard")
        return pending, nxt.value, f, c

    def solve_rates(self):
        """Per-individual solve rate of the last evaluation (games won / games played) and their mean."""
        rates = np.zeros(self.population, np.float32)
        n = _sz()
        mean = C.c_double()
        check(lib().nwg_read_solve_rates(self.handle, _np_ptr(rates), rates.size, C.byref(n), C.byref(mean)),
              "nwg_read_solve_rates")
        return rates[:n.value], mean.value

    def score_table(self, individual: int) -> np.ndarray:
        """Bytes of the 16-bit score table the last tensor-core evaluation built for one individual."""
        n = _sz()
        check(lib().nwg_read_score_table(self.handle, individual, None, 0, C.byref(n)), "nwg_read_score_table")
        out = np.zeros(n.value, np.uint8)
        check(lib().nwg_read_score_table(self.handle, individual, _np_ptr(out), out.size, C.byref(n)),
              "nwg_read_score_table")
        return out

    def resume(self) -> None:
        """TryResumeGenerationFromCheckpointOnDevice: assemble a restored boundary."""
        check(lib().nwg_checkpoint_resume(self.handle), "nwg_checkpoint_resume")
        self.action_count = self.info().action_count

    def assemble(self) -> None:
        """The second half of advance: breed (and widen/inject) the planned children and swap them in."""
        check(lib().nwg_assemble_prepared(self.handle), "nwg_assemble_prepared")
        self.action_count = self.info().action_count

    def checkpoint(self, seed: int, counts: RuntimeWordCounts, config: AssemblyConfig | None = None,
                   pending: PendingInjection | None = None, post_fitness=None, shard_release=None,
                   history: ShardReleaseHistory | None = None, catalog: np.ndarray | None = None) -> "Checkpoint":
        """prepare, then the pre-breeding boundary as a Checkpoint (the runtime stays prepared)."""
        rec = CheckpointRecord()
        cat = None if catalog is None else np.ascontiguousarray(catalog, np.uint8)
        args = self._boundary_args(seed, counts, config, pending, post_fitness, shard_release, history)
        check(lib().nwg_checkpoint_capture(*args, _np_ptr(cat), 0 if cat is None else len(cat), C.byref(rec)),
              "nwg_checkpoint_capture")
        return Checkpoint._take(rec)

    def status(self) -> int:
        v = C.c_int()
        check(lib().nwg_read_status(self.handle, C.byref(v)), "nwg_read_status")
        return v.value

    def current_generation(self):
        n = self.population
        slots = np.zeros(n, np.uint32)
        fitness = np.zeros(n, np.float32)
        evals = np.zeros(n, np.uint32)
        has = np.zeros(n, np.uint8)
        count = _sz()
        gen = _sz()
        check(lib().nwg_download_current_generation(self.handle, _np_ptr(slots), _np_ptr(fitness), _np_ptr(evals),
                                                    _np_ptr(has), n, C.byref(count), C.byref(gen)),
              "nwg_download_current_generation")
        k = count.value
        return dict(slots=slots[:k], fitness=fitness[:k], evaluation_counts=evals[:k], has_fitness=has[:k],
                    generation_index=gen.value)

    def download_slot(self, slot: int) -> np.ndarray:
        out = np.zeros(genome_stride_bytes(self.action_count), np.uint8)
        n = _sz()
        check(lib().nwg_download_slot(self.handle, slot, _np_ptr(out), out.nbytes, C.byref(n)), "nwg_download_slot")
        return out

    def upload_slot(self, slot: int, image: np.ndarray) -> None:
        image = np.ascontiguousarray(image).view(np.uint8)
        check(lib().nwg_upload_slot(self.handle, slot, _np_ptr(image), image.nbytes), "nwg_upload_slot")

    def upload_current_generation(self, slots: np.ndarray, generation_index: int = 0) -> None:
        slots = np.ascontiguousarray(slots, np.uint32)
        check(lib().nwg_upload_current_generation(self.handle, _np_ptr(slots), len(slots), generation_index),
              "nwg_upload_current_generation")

    def assembly_plan(self) -> np.ndarray:
        out = np.zeros(2 * self.population, np.uint32)
        n = _sz()
        check(lib().nwg_download_assembly_plan(self.handle, _np_ptr(out), len(out), C.byref(n)),
              "nwg_download_assembly_plan")
        return out[:2 * n.value].reshape(-1, 2)

    def device_slab(self):
        ptr = _vp()
        pitch = _sz()
        check(lib().nwg_device_slab(self.handle, C.byref(ptr), C.byref(pitch)), "nwg_device_slab")
        return ptr.value, pitch.value

    # ---- row bands (nwg_set_band): one population split by grid rows across ranks ----
    def set_band(self, global_rows: int, band_row_first: int, halo_rows: int) -> None:
        check(lib().nwg_set_band(self.handle, global_rows, band_row_first, halo_rows), "nwg_set_band")

    def device_generation(self):
        """(fitness device pointer, has-fitness device pointer, count) of the current generation."""
        f, h, n = _vp(), _vp(), _sz()
        check(lib().nwg_device_generation(self.handle, C.byref(f), C.byref(h), C.byref(n)), "nwg_device_generation")
        return f.value, h.value, n.value

    def band_prepare(self, seed: int, config: AssemblyConfig | None, fitness_all: int, has_all: int) -> None:
        check(lib().nwg_band_prepare(self.handle, seed, C.byref(config) if config else None, fitness_all, has_all),
              "nwg_band_prepare")

    def band_copy_rows(self, band_row: int, rows: int, dst: int, dst_pitch: int) -> None:
        check(lib().nwg_band_copy_rows(self.handle, band_row, rows, dst, dst_pitch), "nwg_band_copy_rows")

    def band_install_halo(self, above: int, below: int, src_pitch: int) -> None:
        check(lib().nwg_band_install_halo(self.handle, above, below, src_pitch), "nwg_band_install_halo")


class Checkpoint:
    """A RuntimeCheckpoint (slab_runtime.hpp:86-117) on the host: the scalar records in `record` (a
    CheckpointRecord whose pointers are kept pointing at the numpy arrays below) and the arrays as numpy."""

    _ARRAYS = (("slot_indices", np.uint32), ("fitness", np.float32), ("evaluation_counts", np.uint32),
               ("has_fitness", np.uint8))

    def __init__(self, record: CheckpointRecord, slot_indices, fitness, evaluation_counts, has_fitness,
                 parent_pairs, live_organisms, live_genomes):
        self.record = record
        self.slot_indices = np.ascontiguousarray(slot_indices, np.uint32)
        self.fitness = np.ascontiguousarray(fitness, np.float32)
        self.evaluation_counts = np.ascontiguousarray(evaluation_counts, np.uint32)
        self.has_fitness = np.ascontiguousarray(has_fitness, np.uint8)
        self.parent_pairs = np.ascontiguousarray(parent_pairs, np.uint32).reshape(-1, 2)
        self.live_organisms = np.ascontiguousarray(live_organisms, np.uint32)
        self.live_genomes = np.ascontiguousarray(live_genomes, np.uint8).reshape(len(self.live_organisms), -1)
        self._bind()

    def _bind(self) -> None:
        r = self.record
        r.individual_count = len(self.slot_indices)
        r.child_count = len(self.parent_pairs)
        r.live_count = len(self.live_organisms)
        for name in ("slot_indices", "fitness", "evaluation_counts", "has_fitness", "parent_pairs", "live_organisms",
                     "live_genomes"):
            setattr(r, name, _np_ptr(getattr(self, name)))

    @classmethod
    def _take(cls, rec: CheckpointRecord) -> "Checkpoint":
        """Copies a library-filled record's arrays into numpy and frees the library's copies."""
        def arr(ptr, n, dt):
            if n == 0 or not ptr:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), (n,)).copy()
        n, k, live = rec.individual_count, rec.child_count, rec.live_count
        stride = rec.slab_layout.slot_stride_bytes
        try:
            out = cls(CheckpointRecord.from_buffer_copy(rec), arr(rec.slot_indices, n, np.uint32),
                      arr(rec.fitness, n, np.float32), arr(rec.evaluation_counts, n, np.uint32),
                      arr(rec.has_fitness, n, np.uint8), arr(rec.parent_pairs, 2 * k, np.uint32),
                      arr(rec.live_organisms, live, np.uint32), arr(rec.live_genomes, live * stride, np.uint8))
        finally:
            lib().nwg_checkpoint_free(C.byref(rec))
        return out

    def checksum(self) -> int:
        self._bind()
        return lib().nwg_checkpoint_checksum(C.byref(self.record))

    def seal(self) -> None:
        """Stores the current checksum (after the fields were edited)."""
        self.record.checksum = self.checksum()

    def write(self, path) -> None:
        self._bind()
        check(lib().nwg_checkpoint_write(C.byref(self.record), str(path).encode()), "nwg_checkpoint_write")

    @classmethod
    def read(cls, path) -> "Checkpoint":
        rec = CheckpointRecord()
        check(lib().nwg_checkpoint_read(str(path).encode(), C.byref(rec)), "nwg_checkpoint_read")
        return cls._take(rec)

    def restore(self) -> Runtime:
        """A new runtime at this checkpoint's boundary; Runtime.resume() (= assemble) continues it."""
        self._bind()
        handle = _vp()
        check(lib().nwg_checkpoint_restore(C.byref(self.record), C.byref(handle)), "nwg_checkpoint_restore")
        return Runtime._adopt(handle)


def identity_hash(counts: RuntimeWordCounts, history: ShardReleaseHistory | None = None,
                  catalog: np.ndarray | None = None) -> int:
    cat = None if catalog is None else np.ascontiguousarray(catalog, np.uint8)
    return lib().nwg_checkpoint_identity_hash(C.byref(counts), C.byref(history) if history else None, _np_ptr(cat),
                                              0 if cat is None else len(cat))


def write_winner_artifact(binary_path, metadata_path, genome: np.ndarray, metadata: WinnerMetadata,
                          catalog: np.ndarray, action_space_path="", timestamp: str | None = None) -> None:
    g = np.ascontiguousarray(genome).view(np.uint8)
    cat = np.ascontiguousarray(catalog, np.uint8)
    check(lib().nwg_winner_artifact_write(str(binary_path).encode(), str(metadata_path).encode(), _np_ptr(g),
                                          C.byref(metadata), _np_ptr(cat), len(cat), str(action_space_path).encode(),
                                          timestamp.encode() if timestamp is not None else None),
          "nwg_winner_artifact_write")


def read_winner_artifact(binary_path, metadata_path) -> dict:
    """TryReadWinnerArtifact: metadata, genome image, action-space words, path and timestamp."""
    m = WinnerMetadata()
    check(lib().nwg_winner_artifact_read(str(binary_path).encode(), str(metadata_path).encode(), C.byref(m), None, 0,
                                         None, None, None, 0, None, 0), "nwg_winner_artifact_read")
    genome = np.zeros(m.genome_byte_count, np.uint8)
    letters = np.zeros((CATALOG_CAPACITY, 5), np.uint8)
    count = _sz()
    path = C.create_string_buffer(4096)
    stamp = C.create_string_buffer(64)
    check(lib().nwg_winner_artifact_read(str(binary_path).encode(), str(metadata_path).encode(), C.byref(m),
                                         _np_ptr(genome), genome.nbytes, _np_ptr(letters), C.byref(count), path,
                                         len(path), stamp, len(stamp)), "nwg_winner_artifact_read")
    return dict(metadata=m, genome=genome, words=letters[:count.value].copy(), action_space_path=path.value.decode(),
                timestamp=stamp.value.decode())


def convergence_sample_plan(organism_count: int, trainable_count: int, run_seed: int, generation: int):
    """MakeSamplePlan (genetic_convergence.hpp:86-119): organism indices, weight indices, (first, second) pairs."""
    org = np.zeros(256, np.uint32)
    w = np.zeros(8192, np.uint32)
    pairs = np.zeros((512, 2), np.uint32)
    n_o, n_w, n_p = _sz(), _sz(), _sz()
    check(lib().nwg_convergence_sample_plan(organism_count, trainable_count, run_seed, generation, _np_ptr(org),
                                            C.byref(n_o), _np_ptr(w), C.byref(n_w), _np_ptr(pairs), C.byref(n_p)),
          "nwg_convergence_sample_plan")
    return org[:n_o.value].copy(), w[:n_w.value].copy(), pairs[:n_p.value].copy()


class SingleModel:
    """A single-model inference runtime (inference/single_model_device_runtime.hpp:22-47): one genome image and its
    own catalog on the device; select() answers a batch of grids in one call."""

    def __init__(self, genome: np.ndarray, catalog: np.ndarray):
        g = np.ascontiguousarray(genome).view(np.uint8)
        cat = np.ascontiguousarray(catalog, np.uint8)
        handle = _vp()
        check(lib().nwg_single_model_create(_np_ptr(g), g.nbytes, _np_ptr(cat), len(cat), C.byref(handle)),
              "nwg_single_model_create")
        self.handle = handle
        self.catalog = cat

    def close(self):
        if self.handle:
            lib().nwg_single_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def select(self, guesses: np.ndarray, feedback: np.ndarray, turns: np.ndarray):
        """guesses, feedback: (n, 6, 5) letter indices / tiles (0 green, 1 yellow, 2 grey); turns: (n,).
        Returns (action indices, scores) as arrays; raises NwgError on a failed grid."""
        guesses = np.ascontiguousarray(guesses, np.uint8).reshape(-1, 6, 5)
        feedback = np.ascontiguousarray(feedback, np.uint8).reshape(-1, 6, 5)
        turns = np.ascontiguousarray(turns, np.uint8)
        n = len(turns)
        out = (SelectedAction * max(n, 1))()
        check(lib().nwg_single_model_select(self.handle, _np_ptr(guesses), _np_ptr(feedback), _np_ptr(turns), n, out),
              "nwg_single_model_select")
        index = np.array([out[i].action_index for i in range(n)], np.int64)
        score = np.array([out[i].score for i in range(n)], np.float32)
        return index, score


def bf16_gemm_nt(a_ptr: int, lda: int, b_ptr: int, ldb: int, c_ptr: int, ldc: int, m: int, n: int, k: int,
                 stream: int = 0) -> None:
    """C[m][n] = A[m][k] . B[n][k]^T on tcgen05 (device pointers; BF16 operands, FP32 output)."""
    check(lib().nwg_bf16_gemm_nt(a_ptr, lda, b_ptr, ldb, c_ptr, ldc, m, n, k, stream or None), "nwg_bf16_gemm_nt")


def descriptors(slab_ptr: int, pitch: int, slots_ptr: int, count: int, probe_letters: np.ndarray,
                probe_feedback: np.ndarray, probe_turns: np.ndarray, scale: float, out_ptr: int,
                stream: int = 0) -> None:
    """Behavioural descriptors of count genomes on 128 probes (probe arrays [128][4][5], [128][4][5], [128])."""
    letters = np.ascontiguousarray(probe_letters, np.uint8)
    fb = np.ascontiguousarray(probe_feedback, np.uint8)
    turns = np.ascontiguousarray(probe_turns, np.uint8)
    check(lib().nwg_descriptors(slab_ptr, pitch, slots_ptr, count, _np_ptr(letters), _np_ptr(fb), _np_ptr(turns),
                                scale, out_ptr, stream or None), "nwg_descriptors")


class Mlp:
    """The surrogate network (nwg_mlp): 8,192 -> 512 -> 128 -> 1, GELU, BF16 products, FP32 masters, Adam."""

    def __init__(self, capacity_rows: int, seed: int = 0, learning_rate: float = 1e-3):
        handle = _vp()
        check(lib().nwg_mlp_create(capacity_rows, seed, learning_rate, C.byref(handle)), "nwg_mlp_create")
        self.handle = handle
        self.count = lib().nwg_mlp_parameter_count()

    def close(self):
        if self.handle:
            lib().nwg_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def parameters(self) -> np.ndarray:
        out = np.zeros(self.count, np.float32)
        check(lib().nwg_mlp_parameters(self.handle, _np_ptr(out), None), "nwg_mlp_parameters")
        return out

    def set_parameters(self, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, np.float32)
        check(lib().nwg_mlp_parameters(self.handle, None, _np_ptr(v)), "nwg_mlp_parameters")

    def forward(self, x_ptr: int, rows: int, y_ptr: int) -> None:
        check(lib().nwg_mlp_forward(self.handle, x_ptr, rows, y_ptr), "nwg_mlp_forward")

    def gradients(self, x_ptr: int, t_ptr: int, rows: int):
        g = np.zeros(self.count, np.float32)
        loss = C.c_float()
        check(lib().nwg_mlp_gradients(self.handle, x_ptr, t_ptr, rows, _np_ptr(g), C.byref(loss)),
              "nwg_mlp_gradients")
        return g, loss.value

    def train_step(self, x_ptr: int, t_ptr: int, rows: int) -> None:
        check(lib().nwg_mlp_train_step(self.handle, x_ptr, t_ptr, rows), "nwg_mlp_train_step")


class Surrogate:
    """Surrogate-screened evolution of a Runtime's population (nwg_surrogate_*)."""

    def __init__(self, runtime: "Runtime", catalog: np.ndarray, config: SurrogateConfig | None = None,
                 secret_pool: np.ndarray | None = None):
        self.config = config or SurrogateConfig()
        cat = np.ascontiguousarray(catalog, np.uint8)
        pool = None if secret_pool is None else np.ascontiguousarray(secret_pool, np.uint32)
        handle = _vp()
        check(lib().nwg_surrogate_create(runtime.handle, C.byref(self.config), _np_ptr(cat), len(cat), _np_ptr(pool),
                                         0 if pool is None else len(pool), C.byref(handle)), "nwg_surrogate_create")
        self.handle = handle
        self.runtime = runtime

    def close(self):
        if self.handle:
            lib().nwg_surrogate_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance(self, seed: int, counts: RuntimeWordCounts, config: AssemblyConfig) -> SurrogateStats:
        st = SurrogateStats()
        check(lib().nwg_surrogate_advance(self.handle, seed, C.byref(counts), C.byref(config), C.byref(st)),
              "nwg_surrogate_advance")
        return st

