"""B200-native multislice 4D-STEM forward model and ptychographic gradient.

A drop-in for the hot path of ptyrodactyl (``ptyrodactyl.multislice``):
``stem_4d``, ``cbed_image`` and ``make_probe`` keep the reference's signatures
and run hand-written sm_100a CUDA through the C-ABI in ``include/ptyro_b200.h``.
"""

from .types import (  # noqa: F401
    STEM4D,
    AtomicSliceData,
    Distribution,
    ReductionMode,
    TRIVIAL,
    TRIVIAL_DISTRIBUTION,
    AxisUpdate,
    combine_axis_updates,
    create_axis_update,
    create_distribution,
    create_ensemble_axes,
    create_trivial_distribution,
    CalibratedArray,
    DetectorConfig,
    EnsembleAxes,
    MicroscopeConfig,
    PotentialSlices,
    ProbeModes,
    create_atomic_slice_data,
    create_calibrated_array,
    create_detector_config,
    create_microscope_config,
    create_potential_slices,
    create_probe_modes,
    create_stem4d,
)
from .reduce import apply_distribution, apply_distributions  # noqa: F401
from .simulations import (  # noqa: F401
    A_BOHR,
    C_LIGHT,
    E_CHARGE,
    H_PLANCK,
    HBAR,
    M0C2_EV,
    M_E,
    MOTT_BETHE_VOLT_ANGSTROM_SQ,
    aberration,
    helmholtz_coupling,
    phase_interaction_parameter,
    relativistic_mass,
    cbed_amplitude,
    cbed_amplitude_from_atoms,
    cbed_image,
    cbed_image_from_atoms,
    decompose_beam_to_modes,
    fft2,
    fourier_calib,
    fourier_coords,
    interaction_sigma,
    make_probe,
    propagation_func,
    relativistic_wavelength_ang,
    shift_beam_fourier,
    transmission_func,
    run_forward,
    slices_from_atoms,
    stem4d_sharded,
    stem_4d,
    stem_4d_frozen_phonon,
    stem_4d_windowed,
)

from .detectors import (  # noqa: F401
    annular_detector,
    annular_mask,
    clip_cbed,
    stem_4d_clipped,
    stem_4d_annular,
    stem_4d_detectors,
    virtual_detectors,
)
from .autodiff import Stem4dFunction, jvp, make_probe_differentiable, stem_4d_patterns, vjp  # noqa: F401
from . import jacobian  # noqa: F401
from .checked import (  # noqa: F401
    CheckedValueError,
    checked_cbed_image,
    checked_make_probe,
    checked_stem4d_sharded,
    checked_stem_4d,
)
from . import multislice_recon  # noqa: F401
from .multislice_recon import (  # noqa: F401
    multi_slice_multi_modal,
    single_slice_multi_modal,
    single_slice_poscorrected,
    single_slice_ptychography,
)
from .crystal import CrystalData, create_crystal_data, crystal_potential_slices  # noqa: F401
from .elements import kirkland_parameters, lobato_parameters, single_atom_potential  # noqa: F401
from .form_factors import (  # noqa: F401
    KirklandParameters,
    LobatoParameters,
    atomic_form_factor,
    bessel_kv,
    create_kirkland_parameters,
    create_lobato_parameters,
    kirkland_form_factor,
    kirkland_projected_potential,
    lobato_bandlimited_peak,
    lobato_form_factor,
    lobato_projected_potential,
    projected_atom_potential,
)
from .multislice_recon import OPTIMIZERS  # noqa: F401
from .hdf5 import HDF5SchemaError, load_from_h5, save_to_h5  # noqa: F401
from .ensemble import (  # noqa: F401
    bind_cbed_axes,
    coherence_to_distribution,
    ensemble_axes_for_cbed,
    position_jitter_to_distribution,
    probe_modes_to_distribution,
)

__version__ = "0.1.0"
