! Replacement for the reference's module timeloopMod (src/timeloopMod.f90):
! the same module name and the same public subroutine
!
!     subroutine timeloop3D(par, myrank)      ! called from program_solver.f90:71
!
! with the element loop, the Runge-Kutta stages, the sources, the receivers and
! the NPML energy trigger (src/timeloopMod.f90:357-589) run by libnexd.so on one
! GPU through the C-ABI of include/nexd.h (module nexd_capi, nexd_capi.f90).
!
! Kept from the reference: readMesh / readSrc / readRec, prepareSources, the
! receiver interpolation weights, PMLPreCalculation (src/timeloopMod.f90:
! 137-300) and the writers of out/seismo.* and out/energy (591-641).  The host
! hands the library FP64 copies of its arrays (the library rounds them once to
! FP32, the reference's CUSTOM_REAL), one value per element for the per-node
! geometry of the affine tetrahedra (mesh%rx(mesh%ibool(1,ie)) ...), one
! fscale per face, and the source time functions plotstf(:,2,:) exactly as
! the reference's source term uses them (one sample per step, its moment
! sources already differentiated by prepareSources).
!
! A partitioned mesh (par%nproc > 1, one rank per GPU) keeps the mesher's
! interface arrays: the faces the reference marks neighbor = -1 become
! NEXD_FACE_PARTITION faces, mpi_neighbor / mpi_ninterface / mpi_connection /
! mpi_ibool / mpi_ibt fill the halo descriptor of nexd_create_partition, and
! every rank trades one halo export per neighbour with MPI_Sendrecv before the
! loop; the per-stage exchange of SendRecVar (src/mpiMod.f90:310-351) then
! runs inside the library (peer stores over NVLink).
!
! Differences, each stated where it applies: the NPML energy trigger sums the
! energy of one partition, so it is armed only when par%nproc = 1; the NPML
! auxiliary update uses each element's own flux (the reference applies the
! last element's flux to every PML element, src/rungekuttaMod.f90:52-63);
! movie frames are not written (nexd_movie gives the element means that
! collectMovie computes from them).  Errors stop with the library's message,
! as the reference's error paths do.
!
! Build: compile nexd_capi.f90 and this file with the reference's other
! modules in place of its timeloopMod.f90, and link libnexd.so
! (e.g. mpif90 ... nexd_capi.f90 timeloopMod_nexd.f90 ... -L<lib> -lnexd).
! No Fortran compiler exists in this build image, so this file is shipped as
! source; the C driver harness/nexd_solve.c runs the same entry points on the
! same input files and is tested on a GPU.
module timeloopMod
    use iso_c_binding
    use constantsMod
    use meshMod
    use parameterMod
    use sourceReceiverMod
    use vandermondeMod
    use matrixMod
    use plotMod
    use pmlMod
    use typeMod
    use allocateMod
    use mpiMod
    use mpiincludeMod
    use nexd_capi
    implicit none

contains

    subroutine timeloop3D(par, myrank)
        type(parameterVar) :: par
        integer :: myrank
        type(meshVar) :: mesh
        type(srcVar) :: src
        type(recVar) :: rec
        real(kind=CUSTOM_REAL) :: deltat, f0
        real(kind=CUSTOM_REAL), dimension(Np,Np) :: vdmTinv
        real(kind=CUSTOM_REAL), dimension(1) :: r_v, s_v, t_v
        ! prepareSources / receiver weights / PML profiles, as the reference holds them
        real(kind=CUSTOM_REAL), dimension(:,:), allocatable :: srcInt, recInt
        real(kind=CUSTOM_REAL), dimension(:), allocatable :: t0, recTemp, stf_time
        real(kind=CUSTOM_REAL), dimension(:,:,:), allocatable :: plotstf, Ms
        integer, dimension(:), allocatable :: srcelemv
        real(kind=CUSTOM_REAL), dimension(:), allocatable :: ddx, ddy, ddz, alphax, alphay, alphaz, kx, ky, kz
        integer, dimension(:,:), allocatable :: pmlloc
        logical, dimension(:), allocatable :: pmlcheck
        ! the copies handed to the library (their addresses go into the descriptor)
        type(nexd_desc), target :: d
        real(c_double), dimension(:,:), allocatable, target :: Dr8, Ds8, Dt8, lift8, invmass8
        real(c_double), dimension(:,:), allocatable, target :: metric8, fscale8, ylam8, ymu8
        real(c_double), dimension(:,:,:), allocatable, target :: nn8, ss8, tt8
        real(c_double), dimension(:), allocatable, target :: jac8, rho8, vpu8, vsu8, lam8, mu8, wl8
        real(c_double), dimension(:,:), allocatable, target :: prof8, srcInt8, force8, srcM8, recInt8
        real(c_double), dimension(:,:,:), allocatable, target :: stf8
        integer(c_int32_t), dimension(:,:), allocatable, target :: fmask4, nbr4, face4
        integer(c_int32_t), dimension(:,:,:), allocatable, target :: ibn4
        integer(c_int32_t), dimension(:), allocatable, target :: pml4, srcelem4, srctype4, recelem4
        ! results
        real(c_float), dimension(:,:,:,:), allocatable, target :: traces
        real(c_double), dimension(:), allocatable, target :: energy
        integer(c_int32_t), dimension(1), target :: pml_switch
        ! partition interface (par%nproc > 1)
        type(nexd_halo_desc), target :: h
        type(nexd_halo_export), target :: ex_out, ex_in
        integer(c_int32_t), dimension(:), allocatable, target :: hpeer, hnface, helem, hside, hpidx
        integer(c_int32_t), dimension(:,:), allocatable, target :: hpnode
        integer :: npeer, ntot, ierr, nbytes
        integer, dimension(MPI_STATUS_SIZE) :: mpistat
        type(c_ptr) :: ctx
        integer(c_int) :: st
        integer :: ie, is, i, j, r, c, it, K, nsrc, nrec
        character(len=3), parameter :: xyz = 'xyz', kinds = 'uva'  ! seismo.{x,y,z}.%07d.sd{u,v,a}
        integer, dimension(Np) :: iv
        character(len=256) :: filename, path      ! plotPoints2d takes a character(len=80) name

! load database, sources and receivers (src/timeloopMod.f90:137-159)
        call readMesh(myrank, mesh)
        nsrc = 0
        nrec = 0
        f0 = 0.0
        if (mesh%has_src) then
            call readSrc(myrank, src)
            nsrc = src%nsrc
            f0 = maxval(src%srcf0)
        end if
        if (mesh%has_rec) then
            call readRec(myrank, rec)
            nrec = rec%nrec
        end if
        K = mesh%nelem
        deltat = mesh%dtfactor*par%cfl

! NPML damping profiles and flags (src/timeloopMod.f90:249-254, src/pmlMod.f90:90-165)
        allocate(pmlcheck(K), pml4(K), pmlloc(K,3))
        allocate(ddx(mesh%nglob), ddy(mesh%nglob), ddz(mesh%nglob), alphax(mesh%nglob), alphay(mesh%nglob))
        allocate(alphaz(mesh%nglob), kx(mesh%nglob), ky(mesh%nglob), kz(mesh%nglob))
        pmlcheck = .false.
        if (par%set_pml) then
            call PMLPreCalculation(mesh, par, f0, ddx, ddy, ddz, kx, ky, kz, alphax, alphay, alphaz, pmlloc, pmlcheck, myrank)
            allocate(prof8(mesh%nglob, 9))
            prof8(:,1) = ddx
            prof8(:,2) = ddy
            prof8(:,3) = ddz
            prof8(:,4) = alphax
            prof8(:,5) = alphay
            prof8(:,6) = alphaz
            prof8(:,7) = kx
            prof8(:,8) = ky
            prof8(:,9) = kz
        end if
        pml4 = merge(1, 0, pmlcheck)

! sources (src/timeloopMod.f90:284-288; prepareSources, src/sourceReceiverMod.f90:743-814)
        vdmTinv = transpose(mesh%vdm)
        call invert(vdmTinv)
        allocate(srcelemv(K))
        srcelemv = 0
        if (mesh%has_src) then
            allocate(srcInt(Np,nsrc), t0(nsrc), plotstf(par%nt,2,nsrc), Ms(3,3,nsrc))
            Ms = 0.0
            call prepareSources(mesh, src, par, srcInt, vdmTinv, t0, srcelemv, Ms, plotstf, deltat)
            allocate(srcelem4(nsrc), srctype4(nsrc), srcInt8(Np,nsrc), force8(3,nsrc), srcM8(6,nsrc))
            allocate(stf8(1,par%nt,nsrc))
            srcelem4 = src%srcelem
            srctype4 = src%srctype
            srcInt8 = srcInt
            force8 = src%srcangle_force
            do i = 1, nsrc
                ! Mxx Myy Mzz Mxy Mxz Myz of the symmetrised tensor the source term uses
                srcM8(:,i) = (/ Ms(1,1,i), Ms(2,2,i), Ms(3,3,i), Ms(1,2,i), Ms(1,3,i), Ms(2,3,i) /)
                stf8(1,:,i) = plotstf(:,2,i)
            end do
        end if

! receivers (src/timeloopMod.f90:290-300)
        if (mesh%has_rec) then
            allocate(recInt(Np,nrec), recTemp(Np), recInt8(Np,nrec), recelem4(nrec))
            do i = 1, nrec
                r_v(1) = rec%recrst(1,i)
                s_v(1) = rec%recrst(2,i)
                t_v(1) = rec%recrst(3,i)
                call vdm3D(recTemp, r_v, s_v, t_v)
                recInt(:,i) = matmul(vdmTinv, recTemp)
            end do
            recInt8 = recInt
            recelem4 = rec%recelem
        end if

! operators, geometry, material and connectivity as FP64 / INTEGER(4) copies
        allocate(Dr8(Np,Np), Ds8(Np,Np), Dt8(Np,Np), lift8(Np,4*NpF), invmass8(Np,Np), fmask4(NpF,4))
        Dr8 = mesh%Dr
        Ds8 = mesh%Ds
        Dt8 = mesh%Dt
        lift8 = mesh%lift
        invmass8 = matmul(real(mesh%vdm, c_double), transpose(real(mesh%vdm, c_double)))  ! src/timeloopMod.f90:302
        fmask4 = mesh%fmask
        allocate(metric8(9,K), jac8(K), fscale8(4,K), nn8(3,4,K), ss8(3,4,K), tt8(3,4,K))
        allocate(rho8(K), vpu8(K), vsu8(K), lam8(K), mu8(K), ylam8(nMB,K), ymu8(nMB,K), wl8(nMB))
        allocate(nbr4(4,K), face4(4,K), ibn4(NpF,4,K))
        do ie = 1, K
            iv = mesh%ibool(:,ie)
            j = iv(1)          ! affine element: the same geometric factors on every node
            metric8(:,ie) = (/ mesh%rx(j), mesh%ry(j), mesh%rz(j), mesh%sx(j), mesh%sy(j), mesh%sz(j), &
                               mesh%tx(j), mesh%ty(j), mesh%tz(j) /)
            jac8(ie) = mesh%jacobian(j)
            do is = 1, 4
                fscale8(is,ie) = mesh%fscale(1 + (is-1)*NpF, ie)
            end do
        end do
        nn8 = mesh%nnormal
        ss8 = mesh%stangential
        tt8 = mesh%ttangential
        rho8 = mesh%rho
        vpu8 = mesh%vpu
        vsu8 = mesh%vsu
        lam8 = mesh%lambdau
        mu8 = mesh%muu
        ylam8 = mesh%ylambda
        ymu8 = mesh%ymu
        wl8 = mesh%wl
        nbr4 = mesh%neighbor
        face4 = mesh%face
        ibn4 = mesh%ibn
        if (par%nproc > 1) then
            ! faces shared with another partition (neighbor = -1, src/meshMod.f90:776-784)
            do ie = 1, K
                do is = 1, 4
                    if (mesh%neighbor(is,ie) == -1) then
                        nbr4(is,ie) = 0
                        face4(is,ie) = NEXD_FACE_PARTITION
                    end if
                end do
            end do
            ! the interface of this partition (src/meshMod.f90:1006-1110)
            npeer = mesh%mpi_nn
            allocate(hpeer(max(npeer,1)), hnface(max(npeer,1)))
            if (npeer > 0) then
                hpeer(1:npeer) = mesh%mpi_neighbor(1:npeer)
                hnface(1:npeer) = mesh%mpi_ninterface(1:npeer)
            end if
            ntot = 0
            if (npeer > 0) ntot = sum(hnface(1:npeer))
            allocate(helem(max(ntot,1)), hside(max(ntot,1)), hpidx(max(ntot,1)), hpnode(NpF,max(ntot,1)))
            c = 0
            do i = 1, npeer
                do j = 1, hnface(i)
                    c = c + 1
                    ie = mesh%mpi_connection(i,j,1)
                    is = mesh%mpi_connection(i,j,2)
                    helem(c) = ie
                    hside(c) = is
                    hpidx(c) = mesh%mpi_ibool(is,ie)       ! index of the face in the neighbour's list
                    hpnode(:,c) = mesh%mpi_ibt(:,is,ie)    ! node matching, in the neighbour's face order
                end do
            end do
            h%partition = myrank + 1
            h%npeer = npeer
            h%peer = c_loc(hpeer)
            h%nface = c_loc(hnface)
            h%elem = c_loc(helem)
            h%side = c_loc(hside)
            h%peer_index = c_loc(hpidx)
            h%peer_node = c_loc(hpnode)
        end if

! the descriptor (include/nexd.h: nexd_desc)
        d%abi_version = NEXD_ABI_VERSION
        d%N = ORDER
        d%Np = Np
        d%NpF = NpF
        d%nelem = K
        d%nMB = merge(nMB, 0, par%attenuation)
        d%attenuation = merge(1, 0, par%attenuation)
        d%set_pml = merge(1, 0, par%set_pml)
        d%timeint = par%timeint
        d%nt = par%nt
        d%dt = deltat
        d%init_value = 1d-24                      ! q = 1e-24 (src/timeloopMod.f90:185-189)
        d%Dr = c_loc(Dr8)
        d%Ds = c_loc(Ds8)
        d%Dt = c_loc(Dt8)
        d%lift = c_loc(lift8)
        d%invmass = c_loc(invmass8)
        d%fmask = c_loc(fmask4)
        d%metric = c_loc(metric8)
        d%jacobian = c_loc(jac8)
        d%fscale = c_loc(fscale8)
        d%nnormal = c_loc(nn8)
        d%stangential = c_loc(ss8)
        d%ttangential = c_loc(tt8)
        d%rho = c_loc(rho8)
        d%vpu = c_loc(vpu8)
        d%vsu = c_loc(vsu8)
        d%lambdau = c_loc(lam8)
        d%muu = c_loc(mu8)
        d%ylambda = c_loc(ylam8)
        d%ymu = c_loc(ymu8)
        d%wl = c_loc(wl8)
        d%neighbor = c_loc(nbr4)
        d%face = c_loc(face4)
        d%ibn = c_loc(ibn4)
        d%pmlcheck = c_loc(pml4)
        d%pml_profiles = c_null_ptr
        if (par%set_pml) d%pml_profiles = c_loc(prof8)
        d%nsrc = nsrc
        d%srcelem = c_null_ptr
        d%srctype = c_null_ptr
        d%srcInt = c_null_ptr
        d%srcangle_force = c_null_ptr
        d%srcM = c_null_ptr
        d%stf_per_step = 1                        ! stf(it), constant over the RK stages as in the reference
        d%stf = c_null_ptr
        if (nsrc > 0) then
            d%srcelem = c_loc(srcelem4)
            d%srctype = c_loc(srctype4)
            d%srcInt = c_loc(srcInt8)
            d%srcangle_force = c_loc(force8)
            d%srcM = c_loc(srcM8)
            d%stf = c_loc(stf8)
        end if
        d%nrec = nrec
        d%recelem = c_null_ptr
        d%recInt = c_null_ptr
        if (nrec > 0) then
            d%recelem = c_loc(recelem4)
            d%recInt = c_loc(recInt8)
        end if
        d%nbatch = 1
        d%srcbatch = c_null_ptr

! the time loop (src/timeloopMod.f90:357-589) on the GPU
        if (par%nproc > 1) then
            st = nexd_create_partition(d, h, ctx)
            call nexd_check(c_null_ptr, st)
            ! one halo export per neighbour, traded with that neighbour's rank
            nbytes = int(c_sizeof(ex_out))
            do i = 1, npeer
                st = nexd_halo_export_peer(ctx, int(i-1, c_int32_t), ex_out)
                call nexd_check(ctx, st)
                call MPI_SENDRECV(ex_out, nbytes, MPI_BYTE, hpeer(i)-1, 77, ex_in, nbytes, MPI_BYTE, hpeer(i)-1, 77, &
                                  MPI_COMM_WORLD, mpistat, ierr)
                st = nexd_halo_connect(ctx, int(i-1, c_int32_t), ex_in)
                call nexd_check(ctx, st)
            end do
            call sync_mpi()        ! every partition linked before any writes into a neighbour
        else
            st = nexd_create(d, ctx)
            call nexd_check(c_null_ptr, st)
        end if
        if (par%set_pml .and. par%nproc == 1) then
            ! the reference's STA/LTA trigger with its own energy expression (formula 0)
            st = nexd_pml_trigger(ctx, int(par%avg_window1, c_int32_t), int(par%avg_window2, c_int32_t), &
                                  real(par%sta_lta_trigger, c_double), real(f0, c_double), 0_c_int32_t)
            call nexd_check(ctx, st)
        end if
        if (par%log .and. myrank == 0) write(*,*) "Start timeloop over", K, " elements with dt: ", deltat, " and nt : ", par%nt
        st = nexd_run(ctx, 1_c_int32_t, int(par%nt, c_int32_t))
        call nexd_check(ctx, st)
        allocate(traces(max(nrec,1), par%nt, 9, 1), energy(par%nt))
        traces = 0.0
        energy = 0.d0
        pml_switch = 0
        if (nrec > 0) then
            st = nexd_get_traces(ctx, traces)
            call nexd_check(ctx, st)
        end if
        if (par%set_pml .and. par%nproc == 1) then
            st = nexd_get_energy(ctx, energy, pml_switch)
            call nexd_check(ctx, st)
            if (pml_switch(1) > 0) write(*,*) 'PML was switched off at time step ', pml_switch(1)
        end if
        st = nexd_destroy(ctx)

! seismograms and energy (src/timeloopMod.f90:591-641); the time of step it is
! (it-1)*deltat, as in the reference's own seismograms (simulations/brick/ref,
! first row at t = 0)
        allocate(stf_time(par%nt))
        do it = 1, par%nt
            stf_time(it) = (it-1)*deltat
        end do
        do r = 1, nrec
            do c = 1, 9
                ! component order of nexd_get_traces: u x,y,z; v x,y,z; a x,y,z
                write(filename,"('/seismo.',a1,'.',i7.7,'.sd',a1)") xyz(mod(c-1,3)+1:mod(c-1,3)+1), rec%recnr(r), &
                                                                    kinds((c-1)/3+1:(c-1)/3+1)
                path = trim(outpath)//trim(filename)
                call plotPoints2D(stf_time, real(traces(r,:,c,1), CUSTOM_REAL), path)
            end do
        end do
        if (myrank == 0) then
            path = trim(outpath)//'/energy'
            call plotPoints2D(stf_time, real(energy, CUSTOM_REAL), path)
        end if

        deallocate(traces, energy, stf_time, srcelemv, pmlcheck, pml4, pmlloc)
        deallocate(ddx, ddy, ddz, alphax, alphay, alphaz, kx, ky, kz)
        deallocate(Dr8, Ds8, Dt8, lift8, invmass8, fmask4, metric8, jac8, fscale8, nn8, ss8, tt8)
        deallocate(rho8, vpu8, vsu8, lam8, mu8, ylam8, ymu8, wl8, nbr4, face4, ibn4)
        if (allocated(prof8)) deallocate(prof8)
        if (allocated(hpeer)) deallocate(hpeer, hnface, helem, hside, hpidx, hpnode)
        if (mesh%has_src) then
            deallocate(srcInt, t0, plotstf, Ms, srcelem4, srctype4, srcInt8, force8, srcM8, stf8)
            call deallocSrcVar(src)
        end if
        if (mesh%has_rec) then
            deallocate(recInt, recTemp, recInt8, recelem4)
            call deallocRecVar(rec)
        end if
        call deallocMeshVar(mesh)
    end subroutine timeloop3D

end module timeloopMod
