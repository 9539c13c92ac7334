"""mgbrain_b200: a B200-native single-GPU simulation core for MGBrain spiking
networks.  The product is the C ABI in include/mgc.h and the C++ API in
include/mgbrain.h, both in mgbrain_b200/lib/libmgbrain_b200.so; this package
binds the C ABI for Python callers (tests, benchmarks)."""
from .capi import (ACC_FIXED, ACC_FLOAT, LIF, LIF0, LIFB, LIFE, MODE_AUTO, MODE_PUSH, POISSON, RAW,  # noqa: F401
                   MgcError, RULE_ALL, RULE_ALL_BUT_SELF, RULE_FIXED_INDEGREE, RULE_ONE, RULE_PROB,
                   MODE_DEFERRED, MODE_PULL, SCHED_LEARNED, SCHED_STATIC, SCHED_THRESHOLD, Simulator,
                   effective_steps, fault_inject_alloc, lib, measure_scatter, mlp_gradient,
                   selftest_wait_timeout)

__all__ = ["Simulator", "MgcError", "effective_steps", "lib", "measure_scatter", "mlp_gradient", "RAW", "LIF0",
           "POISSON", "LIF", "LIFE", "LIFB", "MODE_AUTO", "MODE_PUSH", "MODE_DEFERRED", "MODE_PULL",
           "SCHED_STATIC", "SCHED_THRESHOLD", "SCHED_LEARNED", "fault_inject_alloc", "selftest_wait_timeout",
           "ACC_FLOAT", "ACC_FIXED", "RULE_PROB", "RULE_ALL", "RULE_ONE", "RULE_ALL_BUT_SELF",
           "RULE_FIXED_INDEGREE"]
