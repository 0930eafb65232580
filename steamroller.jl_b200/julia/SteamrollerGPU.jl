"""
    SteamrollerGPU

Drop-in GPU field solve for Steamroller.jl.  `using SteamrollerGPU` after
`using Steamroller` adds more specific methods of `Steamroller.vcycle!` and
`Steamroller.fmg!` for the supported combination

    ScalarBlockField{2,16,2,Float64} (contiguous storage),
    LaplacianDiscretization{2,2} / HelmholtzDiscretization{2,2} /
    LaplacianDiscretization{2,4} (poisson_order = 4, on its BoxStencil connectivity),
    and in 3D ScalarBlockField{3,16,2,Float64} with LaplacianDiscretization{3,2},
    HelmholtzDiscretization{3,2} or LaplacianDiscretization{3,4} (CartesianGeometry),
    CartesianGeometry / CylindricalGeometry{1} / CylindricalGeometry{2},
    GeneralHomogeneousBoundaryConditions{2},

so `run_from_input(file)` runs unchanged and every Poisson and photoionization solve
(src/streamer.jl:322-334, src/photo.jl:54-57, src/freebc.jl:67-79) goes through
libsrmg.  Any other combination dispatches to the original Julia methods.

Knobs (no input-file keys are needed): `SteamrollerGPU.configure!(; device=0,
enabled=true)`, or the environment variables SRMG_DEVICE and SRMG_DISABLE=1.
"""
module SteamrollerGPU

using Steamroller
using Steamroller: ScalarBlockField, VectorBlockField, LaplacianDiscretization, HelmholtzDiscretization,
    CartesianGeometry, CylindricalGeometry, GeneralHomogeneousBoundaryConditions,
    Neighbor, Boundary, RefBoundary, Child, Tree, NetIonization, FreeBC
using StaticArrays: SVector

const libsrmg = get(ENV, "SRMG_LIB", joinpath(@__DIR__, "..", "srmg", "libsrmg.so"))

const SRMG_OK = Cint(0)

mutable struct State
    ctx::Ptr{Cvoid}
    device::Int
    enabled::Bool
    fingerprint::UInt64
    generation::UInt64
    levelfp::Vector{UInt64}   # per-level fingerprints of the uploaded tree
    fbc::UInt64               # objectid of the FreeBC whose kernel the library holds (0: none)
end

const STATE = State(C_NULL, parse(Int, get(ENV, "SRMG_DEVICE", "0")),
                    get(ENV, "SRMG_DISABLE", "0") != "1", 0, 0, UInt64[], 0)

function configure!(; device=STATE.device, enabled=STATE.enabled)
    if device != STATE.device && STATE.ctx != C_NULL
        ccall((:srmg_destroy, libsrmg), Cvoid, (Ptr{Cvoid},), STATE.ctx)  # also unregisters
        empty!(REGISTERED)
        STATE.ctx = C_NULL
        STATE.fingerprint = 0
        STATE.fbc = 0
    end
    if device != STATE.device && STATE3.ctx != C_NULL
        ccall((:srmg_destroy, libsrmg), Cvoid, (Ptr{Cvoid},), STATE3.ctx)
        STATE3.ctx = C_NULL
        STATE3.fingerprint = 0
    end
    STATE.device = device
    STATE.enabled = enabled
    nothing
end

function check(rc)
    rc == SRMG_OK && return nothing
    msg = unsafe_string(ccall((:srmg_last_error, libsrmg), Cstring, (Ptr{Cvoid},), STATE.ctx))
    error("libsrmg error $rc: $msg")
end

function context()
    if STATE.ctx == C_NULL
        r = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:srmg_create, libsrmg), Cint, (Ptr{Ptr{Cvoid}}, Cint, Cint, Cint, Cint),
                   r, 2, 16, 2, STATE.device)
        rc == SRMG_OK || error("srmg_create failed ($rc)")
        STATE.ctx = r[]
    end
    STATE.ctx
end

# A fingerprint of the tree: refine!/connectivity! (src/streamer.jl:545-549) change
# at least one level's block set or block numbering, so a hash of every level's pairs,
# in order, decides whether the device copy of the tree is stale.  FNV-1a over the
# sequence (coord1, coord2, blk) of each pair: swapping the block ids of two
# coordinates, or moving a pair, changes it.  `invalidate!()` forces the next upload.
@inline fnv(h::UInt64, x) = (h ⊻ (reinterpret(UInt64, Int64(x)))) * 0x100000001b3

function layer_fingerprint(layer)
    h = fnv(0xcbf29ce484222325, length(layer.pairs))
    for (c, blk) in layer.pairs
        h = fnv(fnv(fnv(h, c[1]), c[2]), blk)
    end
    h
end

"""
    invalidate!()

Forget the uploaded tree, so that the next solve uploads the tree and connectivity
again (for callers that rebuild the tree in place in a way the fingerprint might not
see)."""
invalidate!() = (STATE.fingerprint = 0; STATE3.fingerprint = 0; nothing)

# Host ranges page-locked for the fields passed to srmg_vcycle / srmg_fmg, keyed by the
# ElasticArray object: when newblock! resizes a field (src/blockfield.jl:255-260) its
# data moves, so the old range is unregistered before the new one is registered.
const REGISTERED = Dict{UInt64, Tuple{Ptr{Cvoid}, Int}}()

function register!(f)
    ptr, n = Ptr{Cvoid}(pointer(f.u)), sizeof(f.u)
    key = objectid(f.u)
    old = get(REGISTERED, key, nothing)
    old == (ptr, n) && return nothing
    if old !== nothing
        # the old range may already be gone: the result is not checked
        ccall((:srmg_host_unregister, libsrmg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), context(), old[1])
        delete!(REGISTERED, key)
    end
    rc = ccall((:srmg_host_register, libsrmg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Int64), context(), ptr, n)
    rc == SRMG_OK && (REGISTERED[key] = (ptr, n))  # unregistered ranges still work, staged
    nothing
end

function fingerprint(tree)
    h = UInt64(length(tree))
    for layer in tree
        h = h * 0x100000001b3 + layer_fingerprint(layer)
    end
    h
end

function upload!(tree, conn)
    fp = fingerprint(tree)
    fp == STATE.fingerprint && return nothing
    nlev = length(tree)
    npairs = Int64[length(l.pairs) for l in tree]
    pairs = Ptr{Cvoid}[pointer(l.pairs) for l in tree]
    lens(v) = Int64[length(x) for x in v]
    ptrs(v) = Ptr{Cvoid}[pointer(x) for x in v]
    STATE.generation += 1
    GC.@preserve tree conn begin
        check(ccall((:srmg_set_tree, libsrmg), Cint,
                    (Ptr{Cvoid}, Cint, Ptr{Int64}, Ptr{Ptr{Cvoid}}, Ptr{Int64}, Ptr{Ptr{Cvoid}},
                     Ptr{Int64}, Ptr{Ptr{Cvoid}}, Ptr{Int64}, Ptr{Ptr{Cvoid}}, Ptr{Int64},
                     Ptr{Ptr{Cvoid}}, UInt64),
                    context(), nlev, npairs, pairs,
                    lens(conn.neighbor), ptrs(conn.neighbor),
                    lens(conn.boundary), ptrs(conn.boundary),
                    lens(conn.refboundary), ptrs(conn.refboundary),
                    lens(conn.child), ptrs(conn.child), STATE.generation))
    end
    STATE.fingerprint = fp
    STATE.levelfp = UInt64[layer_fingerprint(l) for l in tree]
    nothing
end

geomcode(::CartesianGeometry) = Cint(0)
geomcode(::CylindricalGeometry{1}) = Cint(1)
geomcode(::CylindricalGeometry{2}) = Cint(2)
opcode(::LaplacianDiscretization{2,2}) = (Cint(0), 0.0)
opcode(h::HelmholtzDiscretization{2,2}) = (Cint(1), Float64(h.k2))
opcode(::LaplacianDiscretization{2,4}) = (Cint(2), 0.0)

const GPUField = ScalarBlockField{2,16,2,Float64}
const GPUGeom = Union{CartesianGeometry, CylindricalGeometry{1}, CylindricalGeometry{2}}
const GPUDisc = Union{LaplacianDiscretization{2,2}, HelmholtzDiscretization{2,2}, LaplacianDiscretization{2,4}}

function Steamroller.vcycle!(u::GPUField, b::GPUField, r::GPUField, u1::GPUField, s,
                             tree, conn, geometry::GPUGeom,
                             bc::GeneralHomogeneousBoundaryConditions{2}, lpldisc::GPUDisc;
                             lmax=0, ndown=3, ntop=5, nup=3, ω=1.0)
    if !STATE.enabled
        return invoke(Steamroller.vcycle!, Tuple{Any,Any,Any,Any,Any,Any,Any,Any,Any,Any},
                      u, b, r, u1, s, tree, conn, geometry, bc, lpldisc;
                      lmax, ndown, ntop, nup, ω)
    end
    upload!(tree, conn)
    register!(u)
    register!(b)
    op, k2 = opcode(lpldisc)
    a = Ref(bc.a)
    GC.@preserve u b r u1 a begin
        check(ccall((:srmg_vcycle, libsrmg), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64,
                     Float64, Cint, Float64, Cint, Ptr{Int8}, Cint, Cint, Cint, Cint, Float64, Cint),
                    context(), pointer(u.u), pointer(b.u), pointer(r.u), pointer(u1.u),
                    size(u.u, 3), Float64(s), op, k2, geomcode(geometry),
                    Base.unsafe_convert(Ptr{Int8}, a), lmax, ndown, ntop, nup, Float64(ω), 1))
    end
    nothing
end

function Steamroller.fmg!(u::GPUField, b::GPUField, r::GPUField, u1::GPUField, s,
                          tree, conn, geometry::GPUGeom,
                          bc::GeneralHomogeneousBoundaryConditions{2}, lpldisc::GPUDisc;
                          lmax=0, ndown=3, ntop=5, nup=3, ω=1.25)
    if !STATE.enabled
        return invoke(Steamroller.fmg!, Tuple{Any,Any,Any,Any,Any,Any,Any,Any,Any,Any},
                      u, b, r, u1, s, tree, conn, geometry, bc, lpldisc;
                      lmax, ndown, ntop, nup, ω)
    end
    upload!(tree, conn)
    register!(u)
    register!(b)
    op, k2 = opcode(lpldisc)
    a = Ref(bc.a)
    GC.@preserve u b r u1 a begin
        check(ccall((:srmg_fmg, libsrmg), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64,
                     Float64, Cint, Float64, Cint, Ptr{Int8}, Cint, Cint, Cint, Float64),
                    context(), pointer(u.u), pointer(b.u), pointer(r.u), pointer(u1.u),
                    size(u.u, 3), Float64(s), op, k2, geomcode(geometry),
                    Base.unsafe_convert(Ptr{Int8}, a), ndown, ntop, nup, Float64(ω)))
    end
    nothing
end

"""
    solve!(u, b, s, tree, conn, geometry, bc, lpldisc; tol=1e-8, mixed=true)

Solve to `resnorm(u)/‖b‖ <= tol` (mixed: FP32 V-cycles inside FP64 defect
correction).  Not used by `run_from_input`; for callers that want a tolerance.
Returns (cycles, relative residual).
"""
function solve!(u::GPUField, b::GPUField, s, tree, conn, geometry::GPUGeom,
                bc::GeneralHomogeneousBoundaryConditions{2}, lpldisc::GPUDisc;
                tol=1e-8, mixed=true, max_cycles=1000, ndown=2, ntop=4, nup=2, ω=1.0)
    upload!(tree, conn)
    op, k2 = opcode(lpldisc)
    a = Ref(bc.a)
    # srmg_solve_opts / srmg_stats (include/srmg.h)
    opts = (Float64(tol), Cint(max_cycles), Cint(mixed ? 1 : 0), Cint(ndown), Cint(ntop), Cint(nup),
            Float64(ω), Cint(2), Cint(0))
    optsref = Ref(opts)
    stats = Ref((Cint(0), Cint(0), Cint(0), 0.0, 0.0, 0.0, 0.0))
    GC.@preserve u b a optsref stats begin
        check(ccall((:srmg_solve, libsrmg), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Cint, Float64, Cint,
                     Ptr{Int8}, Ptr{Cvoid}, Ptr{Cvoid}),
                    context(), pointer(u.u), pointer(b.u), size(u.u, 3), Float64(s), op, k2,
                    geomcode(geometry), Base.unsafe_convert(Ptr{Int8}, a),
                    Base.unsafe_convert(Ptr{Cvoid}, optsref), Base.unsafe_convert(Ptr{Cvoid}, stats)))
    end
    st = stats[]
    (st[2], st[4])
end

"""
    solve_async!(u, b, s, tree, conn, geometry, bc, lpldisc; tol=1e-8, mixed=true)
    solve_wait!() -> (cycles, relative residual)

`solve!` in two calls: `solve_async!` enqueues the copies of `u` and `b`, the solve and
the copy of `u` back and returns at once, so that Julia code can run meanwhile;
`solve_wait!` waits for them.  `u` and `b` must stay untouched until the wait, and the
context takes no other call in between.  Not used by `run_from_input`.
"""
function solve_async!(u::GPUField, b::GPUField, s, tree, conn, geometry::GPUGeom,
                      bc::GeneralHomogeneousBoundaryConditions{2}, lpldisc::GPUDisc;
                      tol=1e-8, mixed=true, max_cycles=1000, ndown=2, ntop=4, nup=2, ω=1.0)
    upload!(tree, conn)
    op, k2 = opcode(lpldisc)
    a = Ref(bc.a)
    opts = Ref((Float64(tol), Cint(max_cycles), Cint(mixed ? 1 : 0), Cint(ndown), Cint(ntop), Cint(nup),
                Float64(ω), Cint(2), Cint(0)))
    GC.@preserve u b a opts begin
        check(ccall((:srmg_solve_async, libsrmg), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Cint, Float64, Cint,
                     Ptr{Int8}, Ptr{Cvoid}),
                    context(), pointer(u.u), pointer(b.u), size(u.u, 3), Float64(s), op, k2,
                    geomcode(geometry), Base.unsafe_convert(Ptr{Int8}, a),
                    Base.unsafe_convert(Ptr{Cvoid}, opts)))
    end
    nothing
end

function solve_wait!()
    stats = Ref((Cint(0), Cint(0), Cint(0), 0.0, 0.0, 0.0, 0.0))
    GC.@preserve stats begin
        check(ccall((:srmg_solve_wait, libsrmg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}),
                    context(), Base.unsafe_convert(Ptr{Cvoid}, stats)))
    end
    st = stats[]
    (st[2], st[4])
end

# ---- three-dimensional trees: a second context created with D = 3 ----------------------

mutable struct State3
    ctx::Ptr{Cvoid}
    fingerprint::UInt64
    generation::UInt64
    levelfp::Vector{UInt64}
end
const STATE3 = State3(C_NULL, 0, 0, UInt64[])

function context3()
    if STATE3.ctx == C_NULL
        r = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:srmg_create, libsrmg), Cint, (Ptr{Ptr{Cvoid}}, Cint, Cint, Cint, Cint),
                   r, 3, 16, 2, STATE.device)
        rc == SRMG_OK || error("srmg_create(D = 3) failed ($rc)")
        STATE3.ctx = r[]
    end
    STATE3.ctx
end

function check3(rc)
    rc == SRMG_OK && return nothing
    msg = unsafe_string(ccall((:srmg_last_error, libsrmg), Cstring, (Ptr{Cvoid},), STATE3.ctx))
    error("libsrmg error $rc: $msg")
end

function layer_fingerprint3(layer)
    h = fnv(0xcbf29ce484222325, length(layer.pairs))
    for (c, blk) in layer.pairs
        h = fnv(fnv(fnv(fnv(h, c[1]), c[2]), c[3]), blk)
    end
    h
end

function fingerprint3(tree)
    h = UInt64(length(tree))
    for layer in tree
        h = h * 0x100000001b3 + layer_fingerprint3(layer)
    end
    h
end

# srmg_set_tree3 takes the same per-level pointers as srmg_set_tree; the isbits layouts
# of Pair{CartesianIndex{3},Int} and Neighbor{3}/Boundary{3}/RefBoundary{3}/Child{3}
# are the srmg_*3 structs of include/srmg.h.
function upload3!(tree, conn)
    fp = fingerprint3(tree)
    fp == STATE3.fingerprint && return nothing
    lens(v) = Int64[length(x) for x in v]
    ptrs(v) = Ptr{Cvoid}[pointer(x) for x in v]
    STATE3.generation += 1
    GC.@preserve tree conn begin
        check3(ccall((:srmg_set_tree3, libsrmg), Cint,
                     (Ptr{Cvoid}, Cint, Ptr{Int64}, Ptr{Ptr{Cvoid}}, Ptr{Int64}, Ptr{Ptr{Cvoid}},
                      Ptr{Int64}, Ptr{Ptr{Cvoid}}, Ptr{Int64}, Ptr{Ptr{Cvoid}}, Ptr{Int64},
                      Ptr{Ptr{Cvoid}}, UInt64),
                     context3(), length(tree), Int64[length(l.pairs) for l in tree],
                     Ptr{Cvoid}[pointer(l.pairs) for l in tree],
                     lens(conn.neighbor), ptrs(conn.neighbor), lens(conn.boundary), ptrs(conn.boundary),
                     lens(conn.refboundary), ptrs(conn.refboundary), lens(conn.child), ptrs(conn.child),
                     STATE3.generation))
    end
    STATE3.fingerprint = fp
    STATE3.levelfp = UInt64[layer_fingerprint3(l) for l in tree]
    nothing
end

const GPUField3 = ScalarBlockField{3,16,2,Float64}
const GPUDisc3 = Union{LaplacianDiscretization{3,2}, HelmholtzDiscretization{3,2}, LaplacianDiscretization{3,4}}
opcode(::LaplacianDiscretization{3,2}) = (Cint(0), 0.0)
opcode(h::HelmholtzDiscretization{3,2}) = (Cint(1), Float64(h.k2))
opcode(::LaplacianDiscretization{3,4}) = (Cint(2), 0.0)

function Steamroller.vcycle!(u::GPUField3, b::GPUField3, r::GPUField3, u1::GPUField3, s,
                             tree, conn, geometry::CartesianGeometry,
                             bc::GeneralHomogeneousBoundaryConditions{3}, lpldisc::GPUDisc3;
                             lmax=0, ndown=3, ntop=5, nup=3, ω=1.0)
    if !STATE.enabled
        return invoke(Steamroller.vcycle!, Tuple{Any,Any,Any,Any,Any,Any,Any,Any,Any,Any},
                      u, b, r, u1, s, tree, conn, geometry, bc, lpldisc; lmax, ndown, ntop, nup, ω)
    end
    upload3!(tree, conn)
    op, k2 = opcode(lpldisc)
    a = Ref(bc.a)
    GC.@preserve u b r u1 a begin
        check3(ccall((:srmg_vcycle, libsrmg), Cint,
                     (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64,
                      Float64, Cint, Float64, Cint, Ptr{Int8}, Cint, Cint, Cint, Cint, Float64, Cint),
                     context3(), pointer(u.u), pointer(b.u), pointer(r.u), pointer(u1.u), size(u.u, 4),
                     Float64(s), op, k2, Cint(0), Base.unsafe_convert(Ptr{Int8}, a), lmax, ndown, ntop, nup,
                     Float64(ω), 1))
    end
    nothing
end

function Steamroller.fmg!(u::GPUField3, b::GPUField3, r::GPUField3, u1::GPUField3, s,
                          tree, conn, geometry::CartesianGeometry,
                          bc::GeneralHomogeneousBoundaryConditions{3}, lpldisc::GPUDisc3;
                          lmax=0, ndown=3, ntop=5, nup=3, ω=1.25)
    if !STATE.enabled
        return invoke(Steamroller.fmg!, Tuple{Any,Any,Any,Any,Any,Any,Any,Any,Any,Any},
                      u, b, r, u1, s, tree, conn, geometry, bc, lpldisc; lmax, ndown, ntop, nup, ω)
    end
    upload3!(tree, conn)
    op, k2 = opcode(lpldisc)
    a = Ref(bc.a)
    GC.@preserve u b r u1 a begin
        check3(ccall((:srmg_fmg, libsrmg), Cint,
                     (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64,
                      Float64, Cint, Float64, Cint, Ptr{Int8}, Cint, Cint, Cint, Float64),
                     context3(), pointer(u.u), pointer(b.u), pointer(r.u), pointer(u1.u), size(u.u, 4),
                     Float64(s), op, k2, Cint(0), Base.unsafe_convert(Ptr{Int8}, a), ndown, ntop, nup, Float64(ω)))
    end
    nothing
end

# rhs_level! for the 3D order-4 discretisation (src/multigrid.jl:380-388), while the level
# matches the uploaded octree
function Steamroller.rhs_level!(q1::GPUField3, q::GPUField3, layer, ld::LaplacianDiscretization{3,4},
                                geometry::CartesianGeometry)
    lv = layer.level
    if !(STATE.enabled && STATE3.ctx != C_NULL && 1 <= lv <= length(STATE3.levelfp) &&
         layer_fingerprint3(layer) == STATE3.levelfp[lv])
        return invoke(Steamroller.rhs_level!, Tuple{Any,Any,Any,Any,Any}, q1, q, layer, ld, geometry)
    end
    GC.@preserve q1 q begin
        check3(ccall((:srmg_rhs_level, libsrmg), Cint,
                     (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Cint, Cint, Cint),
                     context3(), pointer(q1.u), pointer(q.u), size(q.u, 4), Cint(lv), Cint(2), Cint(0)))
    end
    nothing
end

# ---- stage preparation and post-processing of derivs! (src/streamer.jl:309-351) ------

# These receive no connectivity, so they run on the GPU only while the uploaded tree is
# the one they are given (the solve of the previous stage uploaded it); after a
# refinement they use the Julia methods until the next solve uploads the new tree.
tree_current(tree) = STATE.enabled && STATE.ctx != C_NULL && fingerprint(tree) == STATE.fingerprint

# netcharge!(tree, q, n, chem) (src/streamer.jl:369-373) for the NetIonization chemistry:
# q = -n_e + n_ion on every valid cell, on the GPU (srmg_netcharge).
function Steamroller.netcharge!(tree::Tree, q::GPUField, n::AbstractVector{<:GPUField}, chem::NetIonization)
    if !tree_current(tree) || length(n) != 2
        return invoke(Steamroller.netcharge!, Tuple{Tree,Any,Any,Any}, tree, q, n, chem)
    end
    ne, ni = n[1], n[2]
    GC.@preserve q ne ni begin
        check(ccall((:srmg_netcharge, libsrmg), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64),
                    context(), pointer(q.u), pointer(ne.u), pointer(ni.u), size(q.u, 3)))
    end
    nothing
end

# rhs_level!(q1, q, layer, ld, geometry) (src/multigrid.jl:380-388) for the order-4
# discretisation on the GPU (srmg_rhs_level, bit-exact): the compact right-hand side of
# derivs! (src/streamer.jl:314-318).  Only the layer is given, so it runs on the GPU
# while that level of the uploaded tree has the same blocks.
function Steamroller.rhs_level!(q1::GPUField, q::GPUField, layer, ld::LaplacianDiscretization{2,4},
                                geometry::GPUGeom)
    lv = layer.level
    if !(STATE.enabled && STATE.ctx != C_NULL && 1 <= lv <= length(STATE.levelfp) &&
         layer_fingerprint(layer) == STATE.levelfp[lv])
        return invoke(Steamroller.rhs_level!, Tuple{Any,Any,Any,Any,Any}, q1, q, layer, ld, geometry)
    end
    GC.@preserve q1 q begin
        check(ccall((:srmg_rhs_level, libsrmg), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Cint, Cint, Cint),
                    context(), pointer(q1.u), pointer(q.u), size(q.u, 3), Cint(lv), Cint(2),
                    geomcode(geometry)))
    end
    nothing
end

# Free boundary conditions (FreeBC, src/freebc.jl).  freebc! runs after setfreebc!'s
# homogeneous solve (already on the GPU through vcycle!/fmg!); the library keeps conf.b
# for fill_ghost_free!.  The transform kernel conf.f is handed over once per FreeBC.
function Steamroller.freebc!(q::GPUField, u::GPUField, h, s, tree, conn, conf::FreeBC{2})
    if !STATE.enabled
        return invoke(Steamroller.freebc!, Tuple{ScalarBlockField,ScalarBlockField,Any,Any,Any,Any,FreeBC},
                      q, u, h, s, tree, conn, conf)
    end
    upload!(tree, conn)
    id = objectid(conf)
    if STATE.fbc != id
        root = Int64[size(tree[1].domain)...]
        GC.@preserve root conf begin
            check(ccall((:srmg_freebc_set, libsrmg), Cint,
                        (Ptr{Cvoid}, Cint, Cint, Ptr{Int64}, Ptr{Float64}, Int64),
                        context(), Cint(Steamroller._perpdim(conf)), Cint(conf.level), root,
                        pointer(conf.f), length(conf.f)))
        end
        STATE.fbc = id
    end
    GC.@preserve q u conf begin
        check(ccall((:srmg_freebc, libsrmg), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Float64, Ptr{Float64}),
                    context(), pointer(q.u), pointer(u.u), size(q.u, 3), Float64(h), Float64(s),
                    pointer(conf.b)))
    end
    nothing
end

function Steamroller.fill_ghost_free!(u::GPUField, conf::FreeBC{2}, tree, l)
    if !(tree_current(tree) && STATE.fbc == objectid(conf))
        return invoke(Steamroller.fill_ghost_free!, Tuple{ScalarBlockField,FreeBC,Any,Any}, u, conf, tree, l)
    end
    GC.@preserve u begin
        check(ccall((:srmg_fill_ghost_free, libsrmg), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64, Cint),
                    context(), pointer(u.u), size(u.u, 3), Cint(l)))
    end
    nothing
end

# electric_field!(tree, f, fabs, u, h, t, e0::SVector) (src/multigrid.jl:421-451) on the
# GPU (srmg_electric_field): face fields and |E| of every block, bit-exact.
function Steamroller.electric_field!(tree::Tree, f::VectorBlockField{2,16,2,Float64}, fabs::GPUField,
                                     u::GPUField, h, t, e0::SVector{2})
    if !tree_current(tree)
        return invoke(Steamroller.electric_field!, Tuple{Tree,Any,Any,Any,Any,Any,SVector},
                      tree, f, fabs, u, h, t, e0)
    end
    e0v = Ref((Float64(e0[1]), Float64(e0[2])))
    GC.@preserve f fabs u e0v begin
        check(ccall((:srmg_electric_field, libsrmg), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Ptr{Float64}),
                    context(), pointer(f.u), pointer(fabs.u), pointer(u.u), size(u.u, 3), Float64(h),
                    Base.unsafe_convert(Ptr{Float64}, e0v)))
    end
    nothing
end

end # module
