"""Loader of the engine's native library (agama_b200/_lib/libagama_b200.so) through ctypes.

There is no CPU implementation behind this module: if the library is missing, importing the
engine's classes raises immediately, and every compute call requires a CUDA device.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_lib", "libagama_b200.so")

D = ctypes.POINTER(ctypes.c_double)
L = ctypes.POINTER(ctypes.c_long)
I = ctypes.POINTER(ctypes.c_int)
F = ctypes.POINTER(ctypes.c_float)
VP = ctypes.c_void_p

# name -> (restype, argtypes); kept in the order of include/agama_b200.h
SIGNATURES = {
    "agama_getError": (ctypes.c_char_p, []),
    "agama_createPotential": (VP, [ctypes.c_char_p]),
    "agama_deletePotential": (None, [VP]),
    "agama_evalPotential": (ctypes.c_double, [VP, D, ctypes.c_double, D, D]),
    "agama_createMultipoleFromDensities": (VP, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]),
    "agama_multipoleCoefsFromDensities": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int,
                                                         ctypes.POINTER(ctypes.c_char_p), I, I, D, D, D]),
    "agama_createMultipoleFromCoefs": (VP, [ctypes.c_int, D, ctypes.c_int, D, D]),
    "agama_getPotentialInfo": (ctypes.c_int, [VP, I, I, I, I, I]),
    "agama_inspectMultipoleFile": (ctypes.c_int, [ctypes.c_char_p, I, I, I, I, I]),
    "agama_writePotential": (ctypes.c_int, [ctypes.c_char_p, VP]),
    "agama_writeMultipoleCoefs": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, D, ctypes.c_int, D, D]),
    "agama_evalPotentialMany": (ctypes.c_int, [VP, ctypes.c_long, D, ctypes.c_double, D, D, D]),
    "agama_evalPotentialManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, VP, VP, VP]),
    "agama_evalPotentialCylMany": (ctypes.c_int, [VP, ctypes.c_long, D, ctypes.c_double, D, D, D]),
    "agama_evalPotentialCylManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, VP, VP, VP]),
    "agama_createDensity": (VP, [ctypes.c_char_p]),
    "agama_deleteDensity": (None, [VP]),
    "agama_evalDensity": (ctypes.c_double, [VP, D, ctypes.c_double]),
    "agama_evalDensityMany": (ctypes.c_int, [VP, ctypes.c_long, D, ctypes.c_double, D]),
    "agama_evalDensityManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, VP]),
    "agama_R_circ": (ctypes.c_double, [VP, ctypes.c_double]),
    "agama_R_from_Lz": (ctypes.c_double, [VP, ctypes.c_double]),
    "agama_R_max": (ctypes.c_double, [VP, ctypes.c_double]),
    "agama_findPlanarOrbitExtent": (None, [VP, ctypes.c_double, ctypes.c_double, D, D]),
    "agama_potentialRadiiMany": (ctypes.c_int, [VP, ctypes.c_int, ctypes.c_long, D, D, D, D]),
    "agama_potentialRadiiManyDevice": (ctypes.c_int, [VP, ctypes.c_int, ctypes.c_long, VP, VP, VP, VP, VP]),
    "agama_setOrbitLanesPerOrbit": (ctypes.c_int, [ctypes.c_int]),
    "agama_setOrbitBlockSize": (ctypes.c_int, [ctypes.c_int]),
    "agama_setActionPrecision": (ctypes.c_int, [ctypes.c_int]),
    "agama_setOrbitPrecision": (ctypes.c_int, [ctypes.c_int]),
    "agama_integrateOrbitsTrajectoryManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, ctypes.c_double,
                                                                 ctypes.c_double, ctypes.c_long, ctypes.c_int, VP, VP,
                                                                 VP, VP, VP]),
    "agama_integrateOrbitsTrajectoryMany": (ctypes.c_int, [VP, ctypes.c_long, D, D, ctypes.c_double, ctypes.c_double,
                                                           ctypes.c_long, ctypes.c_int, D, D, L, I]),
    "agama_createTargetDensityClassic": (VP, [ctypes.c_int, ctypes.c_int, ctypes.c_int, D, ctypes.c_double,
                                              ctypes.c_double]),
    "agama_deleteTarget": (None, [VP]),
    "agama_targetNumCoefs": (ctypes.c_int, [VP]),
    "agama_integrateOrbitsTargetManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, ctypes.c_double,
                                                             ctypes.c_double, ctypes.c_long, VP, VP, VP, VP, VP, VP]),
    "agama_integrateOrbitsTargetMany": (ctypes.c_int, [VP, ctypes.c_long, D, D, ctypes.c_double, ctypes.c_double,
                                                       ctypes.c_long, VP, F, D, L, I]),
    "agama_orbitGraphCreate": (VP, [VP, ctypes.c_long, VP, VP, ctypes.c_double, ctypes.c_double, ctypes.c_long,
                                    VP, VP, VP, VP]),
    "agama_orbitGraphLaunch": (ctypes.c_int, [VP, VP]),
    "agama_orbitGraphLanes": (ctypes.c_int, [VP]),
    "agama_orbitGraphBlockSize": (ctypes.c_int, [VP]),
    "agama_orbitGraphDelete": (None, [VP]),
    "agama_integrateOrbitsMany": (ctypes.c_int, [VP, ctypes.c_long, D, D, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_long, D, L, I]),
    "agama_integrateOrbitsManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, ctypes.c_double,
                                                       ctypes.c_double, ctypes.c_long, VP, VP, VP, VP,
                                                       ctypes.c_int, VP]),
    "agama_integrateOrbitsManyDeviceNoAlloc": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, ctypes.c_double,
                                                              ctypes.c_double, ctypes.c_long, VP, VP, VP, VP,
                                                              ctypes.c_int, VP]),
    "agama_measureFP64Throughput": (ctypes.c_int, [D]),
    "agama_actionPhaseTiming": (ctypes.c_int, [ctypes.c_int, D, L]),
    "agama_actionFinderBracketSamples": (ctypes.c_int, [VP, ctypes.c_long, D, F, F, F]),
    "agama_actionFinderTrainBrackets": (ctypes.c_int, [VP, ctypes.c_long, D, ctypes.c_int, ctypes.c_int,
                                                       ctypes.c_float, ctypes.c_ulonglong, F, F]),
    "agama_actionFinderPredictBrackets": (ctypes.c_int, [VP, ctypes.c_long, F, F]),
    "agama_actionFinderUseBrackets": (ctypes.c_int, [VP, ctypes.c_int]),
    "agama_actionFinderBracketStats": (ctypes.c_int, [VP, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
    "agama_actionFinderCountBrackets": (ctypes.c_int, [VP, ctypes.c_int]),
    "agama_mlpCreate": (VP, [ctypes.c_ulonglong]),
    "agama_mlpDelete": (None, [VP]),
    "agama_mlpNumParams": (ctypes.c_int, []),
    "agama_mlpGetParams": (ctypes.c_int, [VP, F, F]),
    "agama_mlpSetParams": (ctypes.c_int, [VP, F, F]),
    "agama_mlpLossGrad": (ctypes.c_int, [VP, ctypes.c_int, F, F, F, F, F]),
    "agama_mlpTrain": (ctypes.c_int, [VP, ctypes.c_long, F, F, F, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                      ctypes.c_ulonglong, F]),
    "agama_mlpPredictDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, VP]),
    "agama_mlpCheck": (ctypes.c_int, [VP]),
    "agama_gemmBf16Device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, VP, VP, VP, ctypes.c_int,
                                            ctypes.c_int, VP]),
    "agama_createActionFinder": (VP, [VP]),
    "agama_getActionFinderTableSizes": (ctypes.c_int, [VP, I, I, I, I, I]),
    "agama_getActionFinderTables": (ctypes.c_int, [VP, D, D, D, D, D, D, D]),
    "agama_deleteActionFinder": (None, [VP]),
    "agama_evalActionsAnglesFrequencies": (None, [VP, D, D, D, D]),
    "agama_evalActionsAnglesFrequenciesStandalone": (None, [VP, ctypes.c_double, D, D, D, D]),
    "agama_createActionFinderFromTables": (VP, [VP, ctypes.c_int, D, ctypes.c_int, D, D, ctypes.c_int, D,
                                                ctypes.c_int, D, ctypes.c_int, D, D]),
    "agama_evalActionsMany": (ctypes.c_int, [VP, ctypes.c_long, D, D, D]),
    "agama_evalActionsManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, VP, VP]),
    "agama_evalActionsStandaloneMany": (ctypes.c_int, [VP, ctypes.c_long, D, D, ctypes.c_double, D]),
    "agama_evalActionsStandaloneManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, ctypes.c_double, VP,
                                                             VP, VP]),
    "agama_evalActionsAnglesFrequenciesMany": (ctypes.c_int, [VP, ctypes.c_long, D, D, D, D]),
    "agama_evalActionsAnglesFrequenciesManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP, VP, VP, VP]),
    "agama_evalActionsAnglesFrequenciesStandaloneMany": (ctypes.c_int, [VP, ctypes.c_long, D, D, ctypes.c_double,
                                                                         D, D, D]),
    "agama_evalActionsAnglesFrequenciesStandaloneManyDevice": (ctypes.c_int, [VP, ctypes.c_long, VP, VP,
                                                                               ctypes.c_double, VP, VP, VP, VP]),
}

_lib = None


def lib():
    """The loaded library, with argument types declared; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(
                "agama_b200 native library not found at %s; build it with `python -m agama_b200.build`" % LIBPATH)
        L_ = ctypes.CDLL(LIBPATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L_, name)
            f.restype = res
            f.argtypes = args
        _lib = L_
    return _lib


def error():
    return lib().agama_getError().decode()


def check(rc):
    if rc != 0:
        raise RuntimeError("agama_b200: " + error())


def ptr(a, t=D):
    """ctypes pointer to a numpy array (None stays None)"""
    return None if a is None else a.ctypes.data_as(t)
