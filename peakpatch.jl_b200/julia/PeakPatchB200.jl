"""
    PeakPatchB200

Julia binding of libppb.so, the B200 implementation of PeakPatch.jl's per-tile
halo-finding path.  It supplies a drop-in `run_tile(cfg; seed)` with the
signature and behaviour of `PeakPatch.Pipeline.run_tile` (src/Pipeline.jl:66)
and `run_multitile(cfg; ntile, seed)` (src/MultiTile.jl:108), and GPU
methods for the stub-level entry points `fill_noise_threefry!`
(src/InitialConditions/RandomField.jl:70), `find_peaks`
(src/HaloFinder/PeakFind.jl:15-79), `peak_find_tile_gpu` and
`analyse_peaks_gpu_cuda_multirf` (the plug-in stubs of src/PeakPatch.jl:
231-253, 341-366) and the multi-resolution split, all through `ccall` into
the C ABI declared in include/ppb.h.  Errors become Julia exceptions carrying
the library's message.

Usage (with PeakPatch.jl loaded for PipelineConfig, read_homeltab, ...):

    using PeakPatch, PeakPatchB200
    cfg = PipelineConfig(TOML.parsefile("config.toml"))
    halos = PeakPatchB200.run_tile(cfg; seed=42)      # Vector{ExtHaloRecord} or Vector{HaloRecord}

Set ENV["PPB_LIBRARY"] to the path of libppb.so (default: next to this file's
parent directory).
"""
module PeakPatchB200

using DelimitedFiles: readdlm
using LinearAlgebra: Symmetric, eigvals

const libppb = get(ENV, "PPB_LIBRARY", joinpath(@__DIR__, "..", "libppb.so"))

const PPB_OK = Int32(0)
const PPB_ERR_CAPACITY = Int32(-7)

# ppb_tile_params (include/ppb.h); field order and types must match the C struct
struct TileParams
    Omx::Float64; OmB::Float64; Omvac::Float64; h::Float64
    n::Int32
    boxsize::Float64
    nbuff::Int32
    z_out::Float64; z_max::Float64
    ievol::Int32
    cenx::Float64; ceny::Float64; cenz::Float64
    ilpt::Int32
    ioutshear::Int32
    wsmooth::Int32
    rmax2rs::Float64
    seed::UInt64
    plain::Int32
    reserved0::Int32
    pk_scale::Float64      # P(k) multiplier (sigma8 rescale (s8 / s8_table)^2); 0 means 1
    reserved::NTuple{4,Int32}
end

mutable struct HaloBuf
    records::Ptr{Float32}
    capacity::Int64
    count::Int64
    nfields::Int32
    RTHLmax::Float32
    npeaks::Int64
end

mutable struct Context
    h::Ptr{Cvoid}
end

function check(ctx::Context, rc::Int32)
    rc == PPB_OK && return nothing
    buf = Vector{UInt8}(undef, 1024)
    ccall((:ppb_last_error, libppb), Int32, (Ptr{Cvoid}, Ptr{UInt8}, Csize_t), ctx.h, buf, length(buf))
    error("libppb error $(rc): " * unsafe_string(pointer(buf)))
end

function Context(device::Integer=0; hbm_budget::Integer=0)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:ppb_ctx_create, libppb), Int32, (Int32, UInt64, Ref{Ptr{Cvoid}}), device, hbm_budget, h)
    rc == PPB_OK || error("ppb_ctx_create failed ($rc): no usable CUDA device?")
    ctx = Context(h[])
    finalizer(c -> (c.h != C_NULL && ccall((:ppb_ctx_destroy, libppb), Int32, (Ptr{Cvoid},), c.h); c.h = C_NULL), ctx)
    return ctx
end

const _ctx = Ref{Union{Nothing,Context}}(nothing)
default_context() = (_ctx[] === nothing && (_ctx[] = Context(0)); _ctx[])

"""Upload the collapse table (read_homeltab output) to the device."""
function set_collapse_table!(ctx::Context, table::Array{Float32,3}, tp)
    nx, ny, nz = size(table)
    check(ctx, ccall((:ppb_set_collapse_table, libppb), Int32,
                     (Ptr{Cvoid}, Ptr{Float32}, Int32, Int32, Int32, Float64, Float64, Float64, Float64, Float64, Float64),
                     ctx.h, table, nx, ny, nz, tp.X1, tp.X2, tp.Y1, tp.Y2, tp.Z1, tp.Z2))
end

"""Upload the P(k) table of a load_pk-style file (2 columns: k, P)."""
function set_pk_table!(ctx::Context, path::AbstractString)
    data = readdlm(path, comments=true)
    k = Float64.(data[:, 1]); P = Float64.(data[:, 2])
    check(ctx, ccall((:ppb_set_pk_table, libppb), Int32, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int32),
                     ctx.h, k, P, length(k)))
end

function tile_params(cfg, seed::Integer; plain::Bool=false, pk_scale::Real=1.0)
    TileParams(cfg.Omx, cfg.OmB, cfg.Omvac, cfg.h, Int32(cfg.n), cfg.boxsize, Int32(cfg.nbuff),
               cfg.z_out, cfg.z_max, Int32(cfg.ievol), cfg.cenx, cfg.ceny, cfg.cenz, Int32(cfg.ilpt),
               Int32(cfg.ioutshear), Int32(cfg.wsmooth), cfg.rmax2rs, UInt64(seed), Int32(plain), Int32(0),
               Float64(pk_scale), ntuple(_ -> Int32(0), 4))
end

# calls `call(hb)` with a record buffer until it is large enough; returns
# the records as HaloRecord / ExtHaloRecord and the filled HaloBuf
function _with_records(ctx::Context, PP, nf::Int, call)
    cap = 1 << 20
    while true
        buf = Vector{Float32}(undef, nf * cap)
        hb = Ref(HaloBuf(pointer(buf), cap, 0, 0, 0f0, 0))
        rc = GC.@preserve buf call(hb)
        if rc == PPB_ERR_CAPACITY
            cap = Int(hb[].count) + 16
            continue
        end
        check(ctx, rc)
        n = Int(hb[].count)
        recs = reshape(buf[1:nf * n], nf, n)
        halos = nf == 33 ? [PP.ExtHaloRecord(recs[:, i]...) for i in 1:n] :
                           [PP.HaloRecord(recs[:, i]...) for i in 1:n]
        return halos, hb[]
    end
end

"""
    run_tile(cfg::PipelineConfig; seed=42, verbose=false, pk_scale=1.0) -> Vector{HaloRecord} or Vector{ExtHaloRecord}

Drop-in for PeakPatch.run_tile: reads cfg.pkfile, cfg.filterfile and
cfg.tabfile, runs the tile on the GPU, writes cfg.fileout (.pksc) and
returns the records in the reference's peak order.  pk_scale multiplies the
power spectrum (a sigma8 rescale is (sigma8 / sigma8_table)^2).
"""
function run_tile(cfg; seed::Integer=42, verbose::Bool=false, pk_scale::Real=1.0, ctx::Context=default_context())
    PP = Base.root_module(Base.__toplevel__, :PeakPatch)
    table, tp = PP.read_homeltab(cfg.tabfile)
    set_collapse_table!(ctx, table, tp)
    set_pk_table!(ctx, cfg.pkfile)
    Rf = Float64[f[3] for f in PP.read_filterbank(cfg.filterfile)]
    params = Ref(tile_params(cfg, seed; pk_scale=pk_scale))
    nf = cfg.ioutshear >= 1 ? 33 : 11
    halos, hb = _with_records(ctx, PP, nf, hb -> ccall((:ppb_run_tile, libppb), Int32,
                                                      (Ptr{Cvoid}, Ref{TileParams}, Ptr{Float64}, Int32, Ref{HaloBuf}),
                                                      ctx.h, params, Rf, length(Rf), hb))
    PP.write_pksc(cfg.fileout, halos, hb.RTHLmax, Float32(cfg.z_out))
    verbose && @info "run_tile (B200): $(length(halos)) halos from $(hb.npeaks) peaks -> $(cfg.fileout)"
    return halos
end

"""
    run_multitile(cfg; ntile, seed=42, tiles=nothing) -> halos

Drop-in for MultiTile.run_multitile(cfg; ntile, seed): fields on the full
periodic grid, the filter bank on it, peaks and shells per tile (lightcone
tiles beyond chi(z_max) dropped); records in tile order.  tiles: optional
vector of (it, jt, kt) to process, in that order.
"""
function run_multitile(cfg; ntile::Integer, seed::Integer=42, tiles=nothing, verbose::Bool=false,
                       ctx::Context=default_context())
    PP = Base.root_module(Base.__toplevel__, :PeakPatch)
    table, tp = PP.read_homeltab(cfg.tabfile)
    set_collapse_table!(ctx, table, tp)
    set_pk_table!(ctx, cfg.pkfile)
    Rf = Float64[f[3] for f in PP.read_filterbank(cfg.filterfile)]
    params = Ref(tile_params(cfg, seed))
    nf = cfg.ioutshear >= 1 ? 33 : 11
    tl = tiles === nothing ? Int32[] : Int32[t[d] for t in tiles for d in 1:3]
    halos, hb = _with_records(ctx, PP, nf, hb -> ccall((:ppb_run_multitile, libppb), Int32,
                                                      (Ptr{Cvoid}, Ref{TileParams}, Ptr{Float64}, Int32, Int32,
                                                       Ptr{Int32}, Int32, Ref{HaloBuf}),
                                                      ctx.h, params, Rf, length(Rf), ntile,
                                                      isempty(tl) ? C_NULL : pointer(tl), length(tl) ÷ 3, hb))
    verbose && @info "run_multitile (B200): $(length(halos)) halos"
    return halos
end

"""GPU fill_noise_threefry!: bit-identical Threefry-2x64-20 Box-Muller noise."""
function fill_noise_threefry!(noise::Array{Float32,3}, n::Int, seed::Integer; ctx::Context=default_context())
    size(noise) == (n, n, n) || throw(DimensionMismatch("noise must be n x n x n"))
    check(ctx, ccall((:ppb_noise_threefry, libppb), Int32, (Ptr{Cvoid}, Ptr{Float32}, Int32, UInt64),
                     ctx.h, noise, n, UInt64(seed)))
    return noise
end

"""GPU find_peaks (same arguments as PeakFind.find_peaks; mask is updated)."""
function find_peaks(delta::Array{Float32,3}, mask::Array{Int8,3}, xbx, ybx, zbx, alatt, nbuff, fcrit, Rsmooth;
                    max_peaks::Int=2000000, ctx::Context=default_context())
    n1, n2, n3 = size(delta)
    cap = max(1, min(max_peaks, (n1 - 2nbuff) * (n2 - 2nbuff) * (n3 - 2nbuff)))
    pi = Vector{Int64}(undef, cap); pj = similar(pi); pk = similar(pi); ipp = similar(pi)
    pd = Vector{Float32}(undef, cap)
    np = Ref{Int64}(0)
    check(ctx, ccall((:ppb_find_peaks, libppb), Int32,
                     (Ptr{Cvoid}, Ptr{Float32}, Ptr{Int8}, Int32, Int32, Int32, Int32, Float32, Int64,
                      Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Float32}, Ref{Int64}),
                     ctx.h, delta, mask, n1, n2, n3, nbuff, Float32(fcrit), max_peaks, pi, pj, pk, ipp, pd, np))
    PP = Base.root_module(Base.__toplevel__, :PeakPatch)
    cen = ((n1 + 1) / 2, (n2 + 1) / 2, (n3 + 1) / 2)
    return [PP.PeakCandidate(pi[q], pj[q], pk[q], ipp[q], xbx + alatt * (pi[q] - cen[1]),
                             ybx + alatt * (pj[q] - cen[2]), zbx + alatt * (pk[q] - cen[3]), pd[q], Float64(Rsmooth))
            for q in 1:np[]]
end

"""
    peak_find_tile_gpu(delta_tile, filters, fcrits, tile_masks_in, xbx, ybx, zbx, alatt, nbuff, wsmooth,
                       ioutshear) -> (peaks, Rf, FcRf, d2Rf, mask)

Method for the plug-in stub of src/PeakPatch.jl:341-366: rfft(delta) once,
then per filter (in the given order) the window, the inverse transform and
the peak search with fcrits[i] and the mask carried across filters.  Peaks
come in (filter, scan) order; `mask` is a new array (tile_masks_in is not
modified), as the reference's method returns.
"""
function peak_find_tile_gpu(delta_tile::AbstractArray{<:Real,3}, filters::AbstractVector,
                            fcrits::AbstractVector{<:Real}, tile_masks_in::AbstractArray{<:Integer,3}, xbx::Real,
                            ybx::Real, zbx::Real, alatt::Real, nbuff::Integer, wsmooth::Integer,
                            ioutshear::Integer; ctx::Context=default_context())
    PP = Base.root_module(Base.__toplevel__, :PeakPatch)
    n = size(delta_tile, 1)
    size(delta_tile) == (n, n, n) || throw(DimensionMismatch("delta_tile must be n x n x n"))
    length(filters) == length(fcrits) || throw(DimensionMismatch("one fcrit per filter"))
    delta = Array{Float32,3}(delta_tile)
    mask = Array{Int8,3}(tile_masks_in)
    Rf = Float64[f[3] for f in filters]
    fc = Float64.(fcrits)
    cap = max(1, n^3 ÷ 40)
    while true
        pi = Vector{Int32}(undef, cap); pj = similar(pi); pk = similar(pi); filt = similar(pi)
        ipp = Vector{Int64}(undef, cap)
        x = Vector{Float64}(undef, cap); y = similar(x); z = similar(x); Rfo = similar(x)
        FcRf = Vector{Float32}(undef, cap); d2Rf = similar(FcRf)
        np = Ref{Int64}(0)
        m = copy(mask)
        rc = ccall((:ppb_peak_find_tile, libppb), Int32,
                   (Ptr{Cvoid}, Ptr{Float32}, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Ptr{Int8}, Float64, Float64,
                    Float64, Float64, Int32, Int32, Int32, Int64, Ptr{Int32}, Ptr{Int32}, Ptr{Int32}, Ptr{Int64},
                    Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float32}, Ptr{Float64}, Ptr{Float32}, Ptr{Int32},
                    Ref{Int64}),
                   ctx.h, delta, n, Rf, fc, length(Rf), m, xbx, ybx, zbx, alatt, nbuff, wsmooth, ioutshear, cap,
                   pi, pj, pk, ipp, x, y, z, FcRf, Rfo, d2Rf, filt, np)
        if rc == PPB_ERR_CAPACITY
            cap = Int(np[])
            continue
        end
        check(ctx, rc)
        c = Int(np[])
        peaks = [PP.PeakCandidate{Float32}(Int(pi[q]), Int(pj[q]), Int(pk[q]), Int(ipp[q]), x[q], y[q], z[q],
                                           FcRf[q], Rfo[q]) for q in 1:c]
        return (peaks=peaks, Rf=Rfo[1:c], FcRf=FcRf[1:c], d2Rf=d2Rf[1:c], mask=m)
    end
end

"""
    analyse_peaks_gpu_cuda_multirf(delta, etax, etay, etaz, eta2x, eta2y, eta2z, batches, stab, ct_table,
                                   X1, X2, Y1, Y2, Z1, Z2, alatt, ZZon; lapd=nothing, mask=nothing,
                                   nbuff=0, growth_tables=nothing, rmax2rs=0.0, fcrit_override=nothing,
                                   threads=128, ct_out_val=-1.0) -> (results, mask)

Method for the plug-in stub of src/PeakPatch.jl:231-253.  `batches` holds
(peaks_i, peaks_j, peaks_k, Rf, ir2min) tuples, or 7-tuples with per-peak
(ZZon_pp, fcrit_pp) (ext/CUDAExt.jl:2327-2334); `stab` is the ShellTables of
precompute_shells(rmax).  Each result is a NamedTuple of per-peak arrays
(RTHL, Fbarx, e_v, p_v, strain_final, eigs, Srb, Sbar, Sbar2, gradpk,
gradpkf, gradpkrf, d2F, zvir_half); `mask` (when given) comes back updated
batch by batch.  threads and ct_out_val are accepted for the signature (the
table's out-of-range value is -1, as in the reference's CPU path).
"""
function analyse_peaks_gpu_cuda_multirf(delta, etax, etay, etaz, eta2x, eta2y, eta2z, batches::AbstractVector,
                                        stab, ct_table::AbstractArray{<:Real,3}, X1::Real, X2::Real, Y1::Real,
                                        Y2::Real, Z1::Real, Z2::Real, alatt::Real, ZZon::Real;
                                        lapd=nothing, mask=nothing, nbuff::Integer=0, growth_tables=nothing,
                                        rmax2rs::Real=0.0, fcrit_override=nothing, threads::Int=128,
                                        ct_out_val::Real=-1.0, ctx::Context=default_context())
    PP = Base.root_module(Base.__toplevel__, :PeakPatch)
    n = size(delta, 1)
    f32(a) = a === nothing ? C_NULL : Array{Float32,3}(a)
    tab = Array{Float32,3}(ct_table)
    nx, ny, nz = size(tab)
    check(ctx, ccall((:ppb_set_collapse_table, libppb), Int32,
                     (Ptr{Cvoid}, Ptr{Float32}, Int32, Int32, Int32, Float64, Float64, Float64, Float64, Float64,
                      Float64), ctx.h, tab, nx, ny, nz, X1, X2, Y1, Y2, Z1, Z2))
    fcrit = fcrit_override !== nothing ? Float64(fcrit_override) :
            growth_tables !== nothing ? PP.RadialShell.fsc_of_z(Float64(ZZon) - 1.0, growth_tables) : 1.686
    nhunt = isqrt(Int(maximum(stab.shell_r2)))
    nb = length(batches)
    boff = zeros(Int64, nb + 1)
    for b in 1:nb
        boff[b + 1] = boff[b] + length(batches[b][1])
    end
    cat(i, T) = T[x for bt in batches for x in bt[i]]
    pi = cat(1, Int32); pj = cat(2, Int32); pk = cat(3, Int32)
    Rf = Float64[bt[4] for bt in batches]
    ir2 = Int64[bt[5] for bt in batches]
    pp = nb > 0 && length(batches[1]) >= 7
    Zpp = pp ? cat(6, Float64) : C_NULL
    fpp = pp ? cat(7, Float64) : C_NULL
    m = mask === nothing ? C_NULL : Array{Int8,3}(mask)
    out = Matrix{Float64}(undef, 31, max(1, boff[end]))
    d, ex, ey, ez = f32(delta), f32(etax), f32(etay), f32(etaz)
    e2x, e2y, e2z, lp = f32(eta2x), f32(eta2y), f32(eta2z), f32(lapd)
    check(ctx, ccall((:ppb_analyse_peaks_multirf, libppb), Int32,
                     (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32},
                      Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Int32, Int32, Int32, Ptr{Int64}, Ptr{Int32},
                      Ptr{Int32}, Ptr{Int32}, Ptr{Float64}, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}, Float64, Float64,
                      Float64, Ptr{Int8}, Int32, Float64, Int32, Ptr{Float64}),
                     ctx.h, d, ex, ey, ez, e2x, e2y, e2z, lp, n, nhunt, nb, boff, pi, pj, pk, Rf, ir2, Zpp, fpp,
                     Float64(ZZon), fcrit, Float64(alatt), m, nbuff, Float64(rmax2rs), Int32(0), out))
    results = Vector{NamedTuple}(undef, nb)
    for b in 1:nb
        r = out[:, boff[b]+1:boff[b+1]]
        strain = reshape(r[9:17, :], 3, 3, :)
        eigs = reduce(hcat, [sort(real(eigvals(Symmetric(strain[:, :, q]))))
                             for q in 1:size(r, 2)]; init=zeros(3, 0))
        results[b] = (RTHL=r[1, :], Fbarx=r[24, :], e_v=r[25, :], p_v=r[26, :], strain_final=strain, eigs=eigs,
                      Srb=r[2, :], Sbar=r[3:5, :], Sbar2=r[6:8, :], gradpk=r[18:20, :], gradpkf=r[28:30, :],
                      gradpkrf=r[21:23, :], d2F=r[31, :], zvir_half=r[27, :])
    end
    return (results=results, mask=m === C_NULL ? nothing : m)
end

"""
    write_catalog_hdf5(path, halos, cosmo; z_max=10.0)

Method for the HDF5 plug-in stub (src/PeakPatch.jl:67; ext/HDF5Ext.jl:47-104)
without libhdf5: the columns x, y, z, ra, dec, redshift, chi, M200m, RTHL,
vx, vy, vz (+ vx2, vy2, vz2, overdensity, e_v, p_v, Rf, zform for
ExtHaloRecord) as Float32 datasets; cosmo supplies Om (total matter), OL, h.
"""
function write_catalog_hdf5(path::AbstractString, halos::AbstractVector, cosmo; z_max::Float64=10.0)
    PP = Base.root_module(Base.__toplevel__, :PeakPatch)
    nf = eltype(halos) <: PP.ExtHaloRecord ? 33 : 11
    rec = isempty(halos) ? Float32[] : collect(reinterpret(Float32, collect(halos)))
    rc = ccall((:ppb_write_catalog_hdf5, libppb), Int32,
               (Cstring, Ptr{Float32}, Int64, Int32, Float64, Float64, Float64, Float64),
               path, rec, length(halos), nf, cosmo.Om, cosmo.OL, cosmo.h, z_max)
    rc == PPB_OK || error("ppb_write_catalog_hdf5 failed ($rc) for $path")
    return nothing
end

# ---- multi-resolution split (src/MultiResolution.jl) ---------------------
# Methods for the reference's GPU plug-in stubs of run_multitile_split
# (src/PeakPatch.jl:255-339) and the driver itself.  `pk` is a P(k) file path
# (or nothing to keep the context's table); kernels are (kernel_fn_id, dim1,
# dim2) tuples with the ids of isolated_convolve_gpu.

"""GPU isolated_convolve_gpu_multi: one zero-padded rfft, then per kernel the
transfer multiply and irfft; one n^3 array per kernel."""
function isolated_convolve_gpu_multi(noise::Array{Float32,3}, pk, boxsize_local, n::Integer;
                                     kernels=[(0, 0, 0), (1, 1, 0), (1, 2, 0), (1, 3, 0)], nshell::Integer=0,
                                     ctx::Context=default_context())
    pk === nothing || set_pk_table!(ctx, pk)
    ks = Int32[k[j] for k in kernels for j in 1:3]
    out = Array{Float32,4}(undef, n, n, n, length(kernels))
    check(ctx, ccall((:ppb_isolated_convolve, libppb), Int32,
                     (Ptr{Cvoid}, Ptr{Float32}, Int32, Float64, Int32, Ptr{Int32}, Int32, Int32, Ptr{Float32}),
                     ctx.h, noise, size(noise, 1), boxsize_local, n, ks, length(kernels), nshell, out))
    return [out[:, :, :, q] for q in 1:length(kernels)]
end

isolated_convolve_gpu(noise, pk, boxsize_local, n; kernel_fn_id=0, dim1=0, dim2=0, nshell=0,
                      ctx::Context=default_context()) =
    isolated_convolve_gpu_multi(noise, pk, boxsize_local, n; kernels=[(kernel_fn_id, dim1, dim2)], nshell=nshell,
                                ctx=ctx)[1]

"""GPU interpolate_to_tile_gpu: Catmull-Rom tricubic interpolation of the
periodic M^3 coarse field at the tile's cells (bit-identical)."""
function interpolate_to_tile_gpu(coarse::Array{Float32,3}, it, jt, kt, nsub, nmesh, N, M;
                                 ctx::Context=default_context())
    out = Array{Float32,3}(undef, nmesh, nmesh, nmesh)
    check(ctx, ccall((:ppb_interpolate_to_tile, libppb), Int32,
                     (Ptr{Cvoid}, Ptr{Float32}, Int32, Int32, Int32, Int32, Int32, Int64, Int32, Ptr{Float32}),
                     ctx.h, coarse, it, jt, kt, nsub, nmesh, N, M, out))
    return out
end

"""GPU compute_2lpt_gpu: tile-local 2LPT displacements [psi2_x, psi2_y, psi2_z]."""
function compute_2lpt_gpu(delta_tile::Array{Float32,3}, nmesh, boxsize_local; ctx::Context=default_context())
    out = Array{Float32,4}(undef, nmesh, nmesh, nmesh, 3)
    check(ctx, ccall((:ppb_compute_2lpt, libppb), Int32, (Ptr{Cvoid}, Ptr{Float32}, Int32, Float64, Ptr{Float32}),
                     ctx.h, delta_tile, nmesh, boxsize_local, out))
    return [out[:, :, :, d] for d in 1:3]
end

"""GPU compute_laplacian_gpu: irfft(k^2 rfft(delta_tile)) with the Nyquist zeroing."""
function compute_laplacian_gpu(delta_tile::Array{Float32,3}, nmesh, boxsize_local; ctx::Context=default_context())
    out = Array{Float32,3}(undef, nmesh, nmesh, nmesh)
    check(ctx, ccall((:ppb_compute_laplacian, libppb), Int32, (Ptr{Cvoid}, Ptr{Float32}, Int32, Float64, Ptr{Float32}),
                     ctx.h, delta_tile, nmesh, boxsize_local, out))
    return out
end

"""
    run_multitile_split(cfg; ntile, seed=42, coarse_factor=0, coarse_grid=0) -> halos

Drop-in for MultiResolution.run_multitile_split(cfg; ntile, seed, coarse_factor,
coarse_grid, use_gpu=true): every stage on the GPU, records in tile order.
"""
function run_multitile_split(cfg; ntile::Integer, seed::Integer=42, verbose::Bool=false, coarse_factor::Integer=0,
                             coarse_grid::Integer=0, ctx::Context=default_context())
    PP = Base.root_module(Base.__toplevel__, :PeakPatch)
    table, tp = PP.read_homeltab(cfg.tabfile)
    set_collapse_table!(ctx, table, tp)
    set_pk_table!(ctx, cfg.pkfile)
    Rf = Float64[f[3] for f in PP.read_filterbank(cfg.filterfile)]
    params = Ref(tile_params(cfg, seed))
    nf = cfg.ioutshear >= 1 ? 33 : 11
    cap = 1 << 20
    while true
        buf = Vector{Float32}(undef, nf * cap)
        hb = Ref(HaloBuf(pointer(buf), cap, 0, 0, 0f0, 0))
        rc = GC.@preserve buf ccall((:ppb_run_multitile_split, libppb), Int32,
                                    (Ptr{Cvoid}, Ref{TileParams}, Ptr{Float64}, Int32, Int32, Int32, Int32,
                                     Ptr{Int32}, Int32, Ref{HaloBuf}),
                                    ctx.h, params, Rf, length(Rf), ntile, coarse_factor, coarse_grid, C_NULL, 0, hb)
        if rc == PPB_ERR_CAPACITY
            cap = Int(hb[].count) + 16
            continue
        end
        check(ctx, rc)
        n = Int(hb[].count)
        recs = reshape(buf[1:nf * n], nf, n)
        verbose && @info "run_multitile_split (B200): $(n) halos"
        return nf == 33 ? [PP.ExtHaloRecord(recs[:, i]...) for i in 1:n] :
                          [PP.HaloRecord(recs[:, i]...) for i in 1:n]
    end
end

end # module PeakPatchB200
