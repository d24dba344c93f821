"""The reference's generation program on one GPU.

run() follows SRC_F/main_ScaRL.f90:25-214 and create_fields (:362-740):
config_ScaRL.txt names the generation method, the output layout flags and
the input deck; extra_config_ScaRL.txt may fix the tile topology; every deck
sample is generated (tiles, partition of unity, overlap sum and marginal
transform fused on the GPU) and written as HDF5 + XDMF with the reference's
file names, layouts, attributes and time labels.  Samples with std_dev = 0
become the reference's constant-field files.
"""
import datetime
import os
import time

import numpy as np

from . import api as S


def _output_name(folder, name, one_file):
    """The sample's file stem: the deck name, or name-YYMMDD_HHMMSS when its
    first file already exists (create_fields, SRC_F/main_ScaRL.f90:408-443)."""
    first = name + ".h5" if one_file else name + "_proc_00000.h5"
    if os.path.exists(os.path.join(folder, first)):
        return name + "-" + datetime.datetime.now().strftime("%y%m%d_%H%M%S")
    return name


def run(config="config_ScaRL.txt", extra_config="extra_config_ScaRL.txt", ctx=None, nb_procs=1,
        generator=S.GEN_DCT, dtype=S.F64, pad_policy=S.PAD_FULL, workdir=None, sem=False):
    """Generate and write every sample of the deck named by config.

    nb_procs stands for mpirun -np (the tile count); generator GEN_DCT in
    FP64 is the reference's active generator, GEN_PADDED the padded periodic
    method (either precision).  Returns a list of dicts, one per sample."""
    t_init = time.perf_counter()
    base = workdir or os.getcwd()
    path = lambda p: p if os.path.isabs(p) else os.path.join(base, p)
    cfg = S.read_config_ScaRL(path(config))
    inp = path(cfg["input_file"].strip().strip('"'))
    folder, samples = S.read_input_SEM(inp) if sem else S.read_input_ScaRL(inp)
    found, topo_in = S.read_extra_config_ScaRL(path(extra_config))
    out_dir = path(folder)
    os.makedirs(out_dir, exist_ok=True)
    own = ctx is None
    if own:
        ctx = S.Context(0)
    done = []
    t_tic = time.perf_counter()
    try:
        for s in samples:
            labels, times = ["Read_input"], [time.perf_counter() - t_tic]
            t_tic = time.perf_counter()
            S.verify_inputs(s, cfg["gen_meth"])
            name = s.name.decode()
            if s.std_dev == 0.0:
                S.write_constant_field_h5(out_dir, name, s.xMinGlob[:], s.xMaxGlob[:], s.avg)
                done.append({"name": name, "constant": True})
                continue
            topo = tuple(int(v) for v in topo_in) if found else None
            np_eff = int(np.prod(topo)) if topo else nb_procs
            lay = S.sample_layout(s, cfg["gen_meth"], np_eff, topo)
            labels.append("Topology")
            times.append(time.perf_counter() - t_tic)
            t_tic = time.perf_counter()
            field, glay = S.generate_sample(ctx, s, generator=generator, dtype=dtype,
                                            nb_procs=np_eff, topo=topo, pad_policy=pad_policy,
                                            gen_meth=cfg["gen_meth"])
            labels.append("Generation")  # spectrum, transforms, blend, marginal: one fused pass
            times.append(time.perf_counter() - t_tic)
            t_tic = time.perf_counter()
            stem = _output_name(out_dir, name, cfg["one_file"])
            if cfg["gen_meth"] == 2:  # the FFT_MPI field is one global tile
                glay = dict(glay, Np=glay["L"], Np_ovlp=np.zeros(3, np.int32),
                            topo=np.ones(3, np.int32), nb_tiles=1)
            labels += ["Write_file", "Total_Wall_time"]
            w0 = time.perf_counter()
            S.write_sample_h5(ctx, out_dir, stem, field, s, glay, cfg["one_file"], cfg["one_hdf_ds"],
                              times=times + [0.0, 0.0], time_labels=labels)
            times += [time.perf_counter() - w0, time.perf_counter() - t_init]
            # the write is one of the timed steps: its time goes in afterwards,
            # as write_time_on_hdf5 reopens the file (SRC_F/write_output.f90:819-911)
            tv = np.array(times)
            if cfg["one_file"]:
                S.h5_overwrite_dataset(os.path.join(out_dir, stem + ".h5"), "times", tv)
            else:
                for r in range(int(glay["nb_tiles"])):
                    S.h5_overwrite_dataset(os.path.join(out_dir, f"{stem}_proc_{r:05d}.h5"), "times",
                                           tv)
            done.append({"name": name, "stem": stem, "layout": glay, "folder": out_dir,
                         "times": dict(zip(labels, times))})
            t_tic = time.perf_counter()
    finally:
        if own:
            ctx.close()
    return done
