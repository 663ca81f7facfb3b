"""anechoic-b200: B200-native (sm_100a) Onsager-corrected SCA annealing engines for Max-Cut / Ising.

Public API (see engine.py for the reference interfaces each one mirrors):
    Instance, complete_pm1, random_kbit, random_graph, torus    instances and generators (instances.py)
    Schedule, Tables, build_tables, make_tables                  schedules -> fixed-point tables
    DeviceInstance, run, run_batch, run_trial, run_trial_bias    GPU engines through the C ABI (libanechoic.so)
    auto_estimate, auto_choice                                   the cost model that picks engine="auto"
"""
from .instances import (Instance, complete_pm1, random_kbit, random_graph, torus, pad_spins, spin_words,
                        sparse_classes_manifest)
from .engine import (Schedule, Tables, build_tables, make_tables, parse_schedule_flag, DeviceInstance, run,
                     run_batch, run_trial, run_trial_bias, RunResult, Result, ResultBias, tdiv, auto_estimate,
                     auto_choice)
from ._lib import AncError, LIB_PATH

__all__ = ["Instance", "complete_pm1", "random_kbit", "random_graph", "torus", "pad_spins", "spin_words",
           "sparse_classes_manifest", "Schedule", "Tables", "build_tables", "make_tables", "parse_schedule_flag",
           "DeviceInstance", "run", "run_batch", "run_trial", "run_trial_bias", "RunResult", "Result", "ResultBias",
           "tdiv", "auto_estimate", "auto_choice", "AncError", "LIB_PATH"]
