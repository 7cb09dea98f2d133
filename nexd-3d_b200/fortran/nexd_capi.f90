! ISO_C_BINDING interface to libnexd.so (include/nexd.h) for a Fortran host.
!
! A replacement timeloop3D (src/timeloopMod.f90:42 in the reference) keeps
! readMesh / readSrc / readRec / prepareSources and the seismogram writers,
! fills nexd_desc with c_loc() of FP64 copies of its arrays (per-element
! slices of the per-node geometry, fscale per face), and replaces the hot
! loop (src/timeloopMod.f90:357-589) by
!
!     st = nexd_create(d, ctx)
!     st = nexd_run(ctx, 1_c_int32_t, par%nt)
!     st = nexd_get_traces(ctx, traces)        ! (nrec, nt, 9, nbatch)
!     st = nexd_destroy(ctx)
!
! Status 0 is success; nexd_last_error returns the message the reference
! would have printed before `stop`.  Indices in the descriptor stay 1-based.
! No Fortran compiler exists in the build image, so this module is shipped as
! source; the same entry points are exercised through ctypes by the tests.
module nexd_capi
  use iso_c_binding
  implicit none

  integer(c_int32_t), parameter :: NEXD_ABI_VERSION = 1
  integer(c_int32_t), parameter :: NEXD_CONTRACT_FP32 = 0, NEXD_CONTRACT_BF16X3 = 1, NEXD_CONTRACT_AUTO = 2
  integer(c_int32_t), parameter :: NEXD_FACE_PARTITION = -3

  type, bind(C) :: nexd_desc
     integer(c_int32_t) :: abi_version, N, Np, NpF, nelem, nMB, attenuation, set_pml, timeint, nt
     real(c_double)     :: dt, init_value
     type(c_ptr) :: Dr, Ds, Dt, lift, invmass, fmask
     type(c_ptr) :: metric, jacobian, fscale, nnormal, stangential, ttangential
     type(c_ptr) :: rho, vpu, vsu, lambdau, muu, ylambda, ymu, wl
     type(c_ptr) :: neighbor, face, ibn
     type(c_ptr) :: pmlcheck, pml_profiles
     integer(c_int32_t) :: nsrc
     type(c_ptr) :: srcelem, srctype, srcInt, srcangle_force, srcM
     integer(c_int32_t) :: stf_per_step
     type(c_ptr) :: stf
     integer(c_int32_t) :: nrec
     type(c_ptr) :: recelem, recInt
     integer(c_int32_t) :: nbatch
     type(c_ptr) :: srcbatch
  end type nexd_desc

  ! a partition's interface (nexd_create_partition): the mesher's
  ! mpi_neighbor / mpi_ninterface / mpi_connection / mpi_ibool / mpi_ibt
  type, bind(C) :: nexd_halo_desc
     integer(c_int32_t) :: partition, npeer
     type(c_ptr) :: peer, nface, elem, side, peer_index, peer_node
  end type nexd_halo_desc

  ! what a neighbour needs to write into this partition, sent as bytes
  type, bind(C) :: nexd_halo_export
     integer(c_int32_t) :: abi_version, device
     integer(c_int64_t) :: pid
     integer(c_int32_t) :: partition, nface, nbatch, nbuf
     integer(c_int64_t) :: ldq, halo_base
     integer(c_int32_t) :: counter_slot, reserved
     integer(c_int64_t) :: q(3), counters
     integer(c_int8_t) :: q_ipc(64,3), counters_ipc(64)
  end type nexd_halo_export

  interface
     integer(c_int) function nexd_create(d, ctx) bind(C, name="nexd_create")
       import :: nexd_desc, c_ptr, c_int
       type(nexd_desc), intent(in) :: d
       type(c_ptr), intent(out) :: ctx
     end function

     integer(c_int) function nexd_create_partition(d, h, ctx) bind(C, name="nexd_create_partition")
       import :: nexd_desc, nexd_halo_desc, c_ptr, c_int
       type(nexd_desc), intent(in) :: d
       type(nexd_halo_desc), intent(in) :: h
       type(c_ptr), intent(out) :: ctx
     end function

     integer(c_int) function nexd_halo_export_peer(ctx, peer, ex) bind(C, name="nexd_halo_export_peer")
       import :: nexd_halo_export, c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: peer
       type(nexd_halo_export), intent(out) :: ex
     end function

     integer(c_int) function nexd_halo_connect(ctx, peer, ex) bind(C, name="nexd_halo_connect")
       import :: nexd_halo_export, c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: peer
       type(nexd_halo_export), intent(in) :: ex
     end function

     integer(c_int) function nexd_run(ctx, it_begin, it_end) bind(C, name="nexd_run")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: it_begin, it_end
     end function

     integer(c_int) function nexd_get_traces(ctx, traces) bind(C, name="nexd_get_traces")
       import :: c_ptr, c_int, c_float
       type(c_ptr), value :: ctx
       real(c_float), intent(out) :: traces(*)
     end function

     integer(c_int) function nexd_get_field(ctx, b, q) bind(C, name="nexd_get_field")
       import :: c_ptr, c_int, c_int32_t, c_float
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: b
       real(c_float), intent(out) :: q(*)
     end function

     integer(c_int) function nexd_set_field(ctx, b, q) bind(C, name="nexd_set_field")
       import :: c_ptr, c_int, c_int32_t, c_float
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: b
       real(c_float), intent(in) :: q(*)
     end function

     integer(c_int) function nexd_step_io(ctx, it, stf_in, traces_out) bind(C, name="nexd_step_io")
       import :: c_ptr, c_int, c_int32_t, c_float
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: it
       real(c_float), intent(in) :: stf_in(*)
       real(c_float), intent(out) :: traces_out(*)
     end function

     integer(c_int) function nexd_pml_trigger(ctx, w1, w2, thr, f0, formula) bind(C, name="nexd_pml_trigger")
       import :: c_ptr, c_int, c_int32_t, c_double
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: w1, w2, formula
       real(c_double), value :: thr, f0
     end function

     integer(c_int) function nexd_get_energy(ctx, energy, pml_switch) bind(C, name="nexd_get_energy")
       import :: c_ptr, c_int, c_int32_t, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: energy(*)
       integer(c_int32_t), intent(out) :: pml_switch(*)
     end function

     integer(c_int) function nexd_set_contraction(ctx, mode) bind(C, name="nexd_set_contraction")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: mode
     end function

     integer(c_int) function nexd_set_boundary_mlp(ctx, params, count, max_reflection) &
          bind(C, name="nexd_set_boundary_mlp")
       import :: c_ptr, c_int, c_int64_t, c_float
       type(c_ptr), value :: ctx
       real(c_float), intent(in) :: params(*)
       integer(c_int64_t), value :: count
       real(c_float), value :: max_reflection
     end function

     integer(c_int) function nexd_last_error(ctx, buf, n) bind(C, name="nexd_last_error")
       import :: c_ptr, c_int, c_char, c_size_t
       type(c_ptr), value :: ctx
       character(kind=c_char), intent(out) :: buf(*)
       integer(c_size_t), value :: n
     end function

     integer(c_int) function nexd_destroy(ctx) bind(C, name="nexd_destroy")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function
  end interface

contains

  ! Stops with the library's message, as the reference's error paths do
  ! (src/mpiMod.f90:287-307).
  subroutine nexd_check(ctx, st)
    type(c_ptr), intent(in) :: ctx
    integer(c_int), intent(in) :: st
    character(kind=c_char) :: buf(1024)
    integer(c_int) :: ignored
    integer :: i
    character(len=1024) :: msg
    if (st == 0) return
    ignored = nexd_last_error(ctx, buf, int(size(buf), c_size_t))
    msg = ' '
    do i = 1, size(buf)
       if (buf(i) == c_null_char) exit
       msg(i:i) = buf(i)
    end do
    write(*,*) 'nexd error ', st, ': ', trim(msg)
    stop
  end subroutine nexd_check

end module nexd_capi
