"""The reference tutorials' projection loops over an engine population: the
batched forms of AfqmcConstraintPath::measureWithProjection
(tutorials/afqmcConstraintPath/source/afqmcConstraintPath.cpp:93-148) and
AfqmcPhaseless::measureWithProjection (tutorials/afqmcPhaseless/source/
afqmcPhaseless.cpp:125-205), with their E_T and background adjustment
(afqmcConstraintPathMeasure.cpp:31-44, afqmcPhaselessMeasure.cpp:36-47).

The engine does the walker work; this module only sequences it: thermalise
with periodic adjustment, then `writeNumber` blocks of
`measureNumberPerWrite` measurements `measureSkipStep` steps apart, each
block's sums appended to the estimator files (records.write_measurement)
when an output directory is given.  With a torch.distributed process group
the energy and background used for the adjustment are summed over ranks,
as the reference's MPISum does.
"""
import os
from dataclasses import dataclass

import numpy as np

from . import records


@dataclass
class ConstraintPathMethod:
    """AfqmcConstraintPathMethod's loop parameters and their defaults
    (afqmcConstraintPathMethod.cpp:155-182)."""
    dt: float = 0.01
    thermalSize: int = 200
    writeNumber: int = 60
    measureNumberPerWrite: int = 2
    measureSkipStep: int = 5
    ETAdjustStep: int = 10
    ETAdjustMaxSize: int = 100


@dataclass
class ConstraintPathBPMethod(ConstraintPathMethod):
    """AfqmcConstraintPathMethod of the back-propagation tutorial: the
    constrained-path parameters plus backPropagationStep
    (tutorials/afqmcConstraintPathBP/source/afqmcConstraintPathMethod.cpp:19-46)."""
    backPropagationStep: int = 40


@dataclass
class PhaselessMethod:
    """AfqmcPhaselessMethod's loop parameters and their defaults
    (afqmcPhaselessMethod.cpp:160-183)."""
    dt: float = 0.01
    thermalSize: int = 200
    writeNumber: int = 60
    measureNumberPerWrite: int = 2
    measureSkipStep: int = 5
    ETAndBackGroundAdjustStep: int = 10
    ETAndBackGroundAdjustMaxSize: int = 100
    ETAndBackGroundGrowthEstimateStep: int = 5
    ETAndBackGroundGrowthEstimateMaxSize: int = 200

    def growth_measurements(self):
        """numberOfGrowthMeasure (afqmcPhaseless.cpp:43-51)."""
        if self.ETAndBackGroundAdjustMaxSize < self.ETAndBackGroundGrowthEstimateMaxSize:
            return ((self.ETAndBackGroundGrowthEstimateMaxSize - self.ETAndBackGroundAdjustMaxSize)
                    // self.ETAndBackGroundGrowthEstimateStep)
        return 0

    def adjustable(self):
        """isETAndBackGroundAdjustable: the run starts in the Taylor one-body
        form and switches to dense propagators once the background is set."""
        return self.ETAndBackGroundAdjustMaxSize > 0 or self.growth_measurements() > 0


def mixed_energy(eng):
    """returnEnergy: sum HNum / sum den over all ranks."""
    m = records.sum_over_ranks(eng.measurement()[:2])
    return m[1] / m[0]


def cholesky_background(eng):
    """returnCholeskyBg (realMaterialMoleculeMeasureFixedSD2sSD2is.cpp:68-82):
    Re(sum choleskyBgNum / sum den) over all ranks."""
    bg, _ = eng.cholesky_nums()
    tot = records.sum_over_ranks(np.concatenate([eng.measurement()[:1], bg]))
    return (tot[1:] / tot[0]).real


def _blocks(eng, method, out_dir, on_block):
    sums = []
    for i in range(method.writeNumber):
        for _ in range(method.measureNumberPerWrite):
            eng.add_mixed_measurement()
            eng.step(method.measureSkipStep)
        sums.append(eng.measurement())
        if out_dir is not None:
            beta = (method.thermalSize + (i + 0.5) * method.measureNumberPerWrite * method.measureSkipStep
                    - 0.5) * method.dt
            rank, _ = records.rank_world()
            if rank == 0:
                with open(os.path.join(out_dir, "beta.dat"), "a") as f:
                    f.write(f"{beta:26.16e}\n")
            records.write_measurement(eng, out_dir)
        if on_block is not None:
            on_block(i, eng)
        eng.reset_measurement()
    return np.array(sums)


def run_constraint_path(eng, method, out_dir=None, on_block=None):
    """measureWithProjection of the constrained-path driver; returns the block
    sums (writeNumber x 5: den, HNum, KNum, VNum, RNum) and ends with the
    closing half step of prepareStop."""
    eng.set_cadence(0, 0)
    eng.reset_measurement()
    eng.project_half(-1)
    for i in range(method.thermalSize):
        if i < method.ETAdjustMaxSize and i % method.ETAdjustStep == 0:
            eng.add_mixed_measurement()
            eng.set_ET(float(mixed_energy(eng).real))
            eng.reset_measurement()
        eng.step(1)
    sums = _blocks(eng, method, out_dir, on_block)
    eng.project_half(+1)
    return sums


def run_constraint_path_bp(eng, method, out_dir=None, on_block=None):
    """measureWithProjection of the back-propagation driver
    (tutorials/afqmcConstraintPathBP/source/afqmcConstraintPath.cpp:115-172):
    thermalise with E_T adjustment, open a back-propagation window, and in the
    blocks measure the back-propagated observe estimator whenever the window
    is full.  The engine must have the observe estimator on.  Returns the
    block sums (writeNumber x 5: den, HNum, KNum, VNum, RNum)."""
    bp, skip = method.backPropagationStep, method.measureSkipStep
    eng.set_cadence(0, 0)
    eng.reset_measurement()
    eng.project_half(-1)
    for i in range(method.thermalSize):
        if i < method.ETAdjustMaxSize and i % method.ETAdjustStep == 0:
            eng.add_mixed_measurement()
            eng.set_ET(float(mixed_energy(eng).real))
            eng.reset_measurement()
        eng.step(1)
    eng.bp_begin(bp, skip)                        # prepareBackPropagation
    if bp >= skip:
        for _ in range(bp):
            eng.step(1)
    sums = []
    for i in range(method.writeNumber):
        for _ in range(method.measureNumberPerWrite):
            for _ in range(method.measureSkipStep):
                active, index = eng.bp_state()
                if active and index == bp:
                    eng.bp_measure()
                eng.step(1)
            if bp < skip:
                eng.bp_begin(bp, skip)
        sums.append(eng.measurement())
        if out_dir is not None:
            rank, _ = records.rank_world()
            beta = (method.thermalSize + (i + 0.5) * method.measureNumberPerWrite * method.measureSkipStep
                    - 0.5) * method.dt
            if rank == 0:
                with open(os.path.join(out_dir, "beta.dat"), "a") as f:
                    f.write(f"{beta:26.16e}\n")
            records.write_measurement(eng, out_dir)
        if on_block is not None:
            on_block(i, eng)
        eng.reset_measurement()
    eng.project_half(+1)
    return np.array(sums)


def run_phaseless(eng, model, method, out_dir=None, on_block=None):
    """measureWithProjection of the phaseless driver.  `model` is the host
    RealMaterialMolecule (inputs.MoleculeInputs): the background it holds is
    updated at each adjustment, and the engine rebuilds its propagators on
    the GPU from that background and the model's K where the reference
    rebuilds them (returnExpMinusAlphaK).  An adjustable run must start the
    engine in the Taylor one-body form; the rebuild switches it to the dense
    propagators."""
    growth = method.growth_measurements()
    adj_max = method.ETAndBackGroundAdjustMaxSize

    def adjust():
        eng.set_ET(float(mixed_energy(eng).real))
        model.bg = cholesky_background(eng)
        eng.update_background_only(model.bg)
        eng.reset_measurement()

    def rebuild():
        eng.rebuild_propagators(model.K)

    eng.set_cadence(0, 0)
    eng.reset_measurement()
    eng.project_half(-1)
    for i in range(method.thermalSize):
        if i < adj_max and i % method.ETAndBackGroundAdjustStep == 0:
            eng.add_mixed_measurement()
            adjust()
        if i == adj_max - 1 and growth == 0:
            rebuild()
        if growth > 0 and adj_max <= i < method.ETAndBackGroundGrowthEstimateMaxSize:
            if (i + 1 - adj_max) % method.ETAndBackGroundGrowthEstimateStep == 0:
                eng.add_mixed_measurement()
            if i == method.ETAndBackGroundGrowthEstimateMaxSize - 1:
                adjust()
                rebuild()
        eng.step(1)
    sums = _blocks(eng, method, out_dir, on_block)
    eng.project_half(+1)
    return sums
