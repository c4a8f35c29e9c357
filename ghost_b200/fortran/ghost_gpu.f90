!=================================================================
! ghost_gpu.f90 -- ISO_C_BINDING interface of libghost_b200 and
! drop-in replacements for GHOST's HD hot-path routines.
!
! MODULE ghost_gpu      : BIND(C) interfaces of include/ghost_b200.h,
!                         one context per run (ghost_gpu_init).
! Drop-in subroutines   : fftp3d_create_plan, fftp3d_destroy_plan,
!                         fftp3d_real_to_complex, fftp3d_complex_to_real
!                         (replacing fftp-3/fftp3D.fpp), and derivk3,
!                         laplak3, rotor3, prodre3, nonlhd3, energy,
!                         helicity, cross, maxabs, spectrumc (replacing
!                         pseudo/pseudospec3D_hd.f90) with GHOST's argument
!                         lists.  Arrays are GHOST's host arrays; the library
!                         stages them through the GPU.  Codes that keep
!                         their fields on the device call the ghost_* C
!                         functions with device pointers directly.
!
! Build (with gfortran >= 9):
!   gfortran -c -cpp ghost_gpu.f90
!   link with -L<repo>/ghost_b200 -lghost_b200 -lcudart
! GHOST's fprecision module supplies GP; GHOST_GP_KIND below must match
! (4 = SINGLE, 8 = DOUBLE).
!=================================================================
      MODULE ghost_gpu
      USE ISO_C_BINDING
      IMPLICIT NONE

      INTEGER(C_INT), PARAMETER :: GHOST_OK = 0
      INTEGER(C_INT), PARAMETER :: GHOST_SINGLE = 4, GHOST_DOUBLE = 8
      TYPE(C_PTR), SAVE :: gctx = C_NULL_PTR

      TYPE, BIND(C) :: ghost_info
         INTEGER(C_INT)    :: nx, ny, nz, precision, anis, nmax, nmaxperp
         REAL(C_DOUBLE)    :: kmax, tiny, Lx, Ly, Lz, Dkx, Dky, Dkz, Dkk
         INTEGER(C_SIZE_T) :: spectral_elems, real_elems
      END TYPE ghost_info

      INTERFACE
       FUNCTION ghost_ctx_create(nx,ny,nz,Lx,Ly,Lz,arbsize,prec,ctx) &
                BIND(C,name="ghost_ctx_create") RESULT(s)
         IMPORT :: C_INT, C_DOUBLE, C_PTR
         INTEGER(C_INT), VALUE :: nx, ny, nz, arbsize, prec
         REAL(C_DOUBLE), VALUE :: Lx, Ly, Lz
         TYPE(C_PTR) :: ctx
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_destroy(ctx) BIND(C,name="ghost_ctx_destroy") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_get_info(ctx,info) BIND(C,name="ghost_ctx_get_info") RESULT(s)
         IMPORT :: C_INT, C_PTR, ghost_info
         TYPE(C_PTR), VALUE :: ctx
         TYPE(ghost_info) :: info
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_set_stream(ctx,stream) BIND(C,name="ghost_ctx_set_stream") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, stream
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_set_kmax(ctx,kmax) BIND(C,name="ghost_ctx_set_kmax") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_DOUBLE), VALUE :: kmax
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_synchronize(ctx) BIND(C,name="ghost_ctx_synchronize") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_set_wait_cap(ctx,cap) BIND(C,name="ghost_ctx_set_wait_cap") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT), VALUE :: cap
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_inject_stall(ctx,enable) BIND(C,name="ghost_ctx_inject_stall") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT), VALUE :: enable
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_launch_count(ctx,n) BIND(C,name="ghost_ctx_launch_count") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_LONG_LONG
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_LONG_LONG) :: n
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_enable_timers(ctx,enable) BIND(C,name="ghost_ctx_enable_timers") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT), VALUE :: enable
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_read_timers(ctx,ms,launches) BIND(C,name="ghost_ctx_read_timers") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE, C_LONG_LONG
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_DOUBLE) :: ms(10)
         INTEGER(C_LONG_LONG) :: launches(10)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_last_error_string() BIND(C,name="ghost_last_error_string") RESULT(p)
         IMPORT :: C_PTR
         TYPE(C_PTR) :: p
       END FUNCTION
       FUNCTION ghost_fftp3d_create_plan(ctx,n,fftdir,flags,plan) &
                BIND(C,name="ghost_fftp3d_create_plan") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT) :: n(3)
         INTEGER(C_INT), VALUE :: fftdir, flags
         TYPE(C_PTR) :: plan
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_fftp3d_destroy_plan(plan) BIND(C,name="ghost_fftp3d_destroy_plan") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: plan
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_fftp3d_real_to_complex(plan,in,out) &
                BIND(C,name="ghost_fftp3d_real_to_complex") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: plan, in, out
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_fftp3d_complex_to_real(plan,in,out) &
                BIND(C,name="ghost_fftp3d_complex_to_real") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: plan, in, out
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_derivk3(ctx,a,b,dir) BIND(C,name="ghost_derivk3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b
         INTEGER(C_INT), VALUE :: dir
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_laplak3(ctx,a,b) BIND(C,name="ghost_laplak3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_rotor3(ctx,a,b,c,dir) BIND(C,name="ghost_rotor3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         INTEGER(C_INT), VALUE :: dir
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_prodre3(ctx,a,b,c,d,e,f) BIND(C,name="ghost_prodre3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_nonlhd3(ctx,a,b,c,g,dir) BIND(C,name="ghost_nonlhd3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b, c, g
         INTEGER(C_INT), VALUE :: dir
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_energy(ctx,a,b,c,d,kin) BIND(C,name="ghost_energy") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         REAL(C_DOUBLE) :: d
         INTEGER(C_INT), VALUE :: kin
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_helicity(ctx,a,b,c,d) BIND(C,name="ghost_helicity") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         REAL(C_DOUBLE) :: d
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_cross(ctx,a,b,c,d,e,f,g,kin) BIND(C,name="ghost_cross") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f
         REAL(C_DOUBLE) :: g
         INTEGER(C_INT), VALUE :: kin
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_divergence(ctx,a,b,c,d) BIND(C,name="ghost_divergence") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         REAL(C_DOUBLE) :: d
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_maxabs(ctx,a,b,c,d,kin) BIND(C,name="ghost_maxabs") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         REAL(C_DOUBLE) :: d
         INTEGER(C_INT), VALUE :: kin
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_spectrumc(ctx,a,b,c,kin,hel,Ek,Hk) BIND(C,name="ghost_spectrumc") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         INTEGER(C_INT), VALUE :: kin, hel
         REAL(C_DOUBLE) :: Ek(*), Hk(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       ! spectra without any allocation (device arrays only; see the C header)
       FUNCTION ghost_spectrumc_noalloc(ctx,a,b,c,kin,hel,Ek,Hk) &
                BIND(C,name="ghost_spectrumc_noalloc") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         INTEGER(C_INT), VALUE :: kin, hel
         REAL(C_DOUBLE) :: Ek(*), Hk(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_hdcheck(ctx,vx,vy,vz,fx,fy,fz,hel,chk,out) BIND(C,name="ghost_hdcheck") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, fx, fy, fz
         INTEGER(C_INT), VALUE :: hel, chk
         REAL(C_DOUBLE) :: out(5)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_normalize(ctx,fx,fy,fz,f0,kin) BIND(C,name="ghost_normalize") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, fx, fy, fz
         REAL(C_DOUBLE), VALUE :: f0
         INTEGER(C_INT), VALUE :: kin
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_sharp(ctx,a,b,delta) BIND(C,name="ghost_sharp") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b
         REAL(C_DOUBLE), VALUE :: delta
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_hd_rkstep1(ctx,vx,vy,vz,C1,C2,C3) BIND(C,name="ghost_hd_rkstep1") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, C1, C2, C3
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_hd_rkstep2(ctx,o,dt,nu,vx,vy,vz,C1,C2,C3,fx,fy,fz) &
                BIND(C,name="ghost_hd_rkstep2") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, C1, C2, C3, fx, fy, fz
         INTEGER(C_INT), VALUE :: o
         REAL(C_DOUBLE), VALUE :: dt, nu
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_hd_run(ctx,nsteps,ord,dt,nu,vx,vy,vz,C1,C2,C3,fx,fy,fz) &
                BIND(C,name="ghost_hd_run") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, C1, C2, C3, fx, fy, fz
         INTEGER(C_INT), VALUE :: nsteps, ord
         REAL(C_DOUBLE), VALUE :: dt, nu
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_advect3(ctx,a,b,c,d,e) BIND(C,name="ghost_advect3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_bouss_rkstep2(ctx,o,dt,nu,kappa,omegaz,xmom,xtemp, &
                vx,vy,vz,th,C1,C2,C3,C20,fx,fy,fz,fs) &
                BIND(C,name="ghost_bouss_rkstep2") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, th, C1, C2, C3, C20
         TYPE(C_PTR), VALUE :: fx, fy, fz, fs
         INTEGER(C_INT), VALUE :: o
         REAL(C_DOUBLE), VALUE :: dt, nu, kappa, omegaz, xmom, xtemp
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_bouss_run(ctx,nsteps,ord,dt,nu,kappa,omegaz,xmom,xtemp, &
                vx,vy,vz,th,fx,fy,fz,fs) BIND(C,name="ghost_bouss_run") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, th, fx, fy, fz, fs
         INTEGER(C_INT), VALUE :: nsteps, ord
         REAL(C_DOUBLE), VALUE :: dt, nu, kappa, omegaz, xmom, xtemp
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_create_batch(nx,ny,nz,nruns,prec,ctx) &
                BIND(C,name="ghost_ctx_create_batch") RESULT(s)
         IMPORT :: C_INT, C_PTR
         INTEGER(C_INT), VALUE :: nx, ny, nz, nruns, prec
         TYPE(C_PTR) :: ctx
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_batch_set_nu(ctx,nu) BIND(C,name="ghost_batch_set_nu") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_DOUBLE) :: nu(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_batch_energy(ctx,a,b,c,kin,out) BIND(C,name="ghost_batch_energy") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: out(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_batch_init_random_solenoidal(ctx,seeds,kdn,kup,shape,amp,ox,oy,oz) &
                BIND(C,name="ghost_batch_init_random_solenoidal") RESULT(s)
         IMPORT :: C_INT, C_INT32_T, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, ox, oy, oz
         INTEGER(C_INT32_T) :: seeds(*)
         REAL(C_DOUBLE), VALUE :: kdn, kup, amp
         INTEGER(C_INT), VALUE :: shape
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_create(ncls,n,nruns,prec,ens) BIND(C,name="ghost_ensemble_create") RESULT(s)
         IMPORT :: C_INT, C_PTR
         INTEGER(C_INT), VALUE :: ncls, prec
         INTEGER(C_INT) :: n(*), nruns(*)
         TYPE(C_PTR) :: ens
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_destroy(ens) BIND(C,name="ghost_ensemble_destroy") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_fields(ens,c,vx,vy,vz) BIND(C,name="ghost_ensemble_fields") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT), VALUE :: c
         TYPE(C_PTR) :: vx, vy, vz
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_class(ens,c,ctx) BIND(C,name="ghost_ensemble_class") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT), VALUE :: c
         TYPE(C_PTR) :: ctx
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_init(ens,seeds,kdn,kupf,shape,amp,nu) BIND(C,name="ghost_ensemble_init") RESULT(s)
         IMPORT :: C_INT, C_INT32_T, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT32_T) :: seeds(*)
         REAL(C_DOUBLE), VALUE :: kdn, kupf, amp
         INTEGER(C_INT), VALUE :: shape
         REAL(C_DOUBLE) :: nu(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_autotune(ens,ord,dt,cfg) BIND(C,name="ghost_ensemble_autotune") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT), VALUE :: ord
         REAL(C_DOUBLE), VALUE :: dt
         INTEGER(C_INT) :: cfg(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_set_mode(ens,multi) BIND(C,name="ghost_ensemble_set_mode") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT), VALUE :: multi
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_get_mode(ens,multi) BIND(C,name="ghost_ensemble_get_mode") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT) :: multi
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_run(ens,nsteps,ord,dt) BIND(C,name="ghost_ensemble_run") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT), VALUE :: nsteps, ord
         REAL(C_DOUBLE), VALUE :: dt
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ensemble_energy(ens,kin,out) BIND(C,name="ghost_ensemble_energy") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ens
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: out(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       ! slab decomposition (GHOST's kx-slab / z-slab layout; the caller runs
       ! the all-to-alls between pack and unpack, e.g. MPI_ALLTOALLV)
       FUNCTION ghost_slab_range(n1,n2,nprocs,irank,ista,iend) BIND(C,name="ghost_slab_range") RESULT(s)
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: n1, n2, nprocs, irank
         INTEGER(C_INT) :: ista, iend
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_create(nx,ny,nz,lx,ly,lz,arbsize,prec,rank,nranks,slab) &
           BIND(C,name="ghost_slab_create") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         INTEGER(C_INT), VALUE :: nx, ny, nz, arbsize, prec, rank, nranks
         REAL(C_DOUBLE), VALUE :: lx, ly, lz
         TYPE(C_PTR) :: slab
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_destroy(slab) BIND(C,name="ghost_slab_destroy") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_layout(slab,ista,nxhl,ksta,nzl) BIND(C,name="ghost_slab_layout") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT) :: ista(*), nxhl(*), ksta(*), nzl(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_rows(slab,rows) BIND(C,name="ghost_slab_rows") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT) :: rows
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_launch_count(slab,count) BIND(C,name="ghost_slab_launch_count") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_LONG_LONG
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_LONG_LONG) :: count
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_set_stream(slab,stream) BIND(C,name="ghost_slab_set_stream") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab, stream
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_synchronize(slab) BIND(C,name="ghost_slab_synchronize") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_hd_front(slab,v,c,copy,prune,w) BIND(C,name="ghost_slab_hd_front") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         TYPE(C_PTR) :: v(3), c(3), w(6)
         INTEGER(C_INT), VALUE :: copy, prune
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_hd_xpass(slab,prune,fin,fout) BIND(C,name="ghost_slab_hd_xpass") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT), VALUE :: prune
         TYPE(C_PTR) :: fin(6), fout(3)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_hd_back(slab,o,dt,nu,prune,w,v,c,f) BIND(C,name="ghost_slab_hd_back") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT), VALUE :: o, prune
         REAL(C_DOUBLE), VALUE :: dt, nu
         TYPE(C_PTR) :: w(3), v(3), c(3), f(3)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_pack(slab,dir,nf,prune,fields,send) BIND(C,name="ghost_slab_pack") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab, send
         INTEGER(C_INT), VALUE :: dir, nf, prune
         TYPE(C_PTR) :: fields(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_unpack(slab,dir,nf,prune,recv,fields) BIND(C,name="ghost_slab_unpack") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab, recv
         INTEGER(C_INT), VALUE :: dir, nf, prune
         TYPE(C_PTR) :: fields(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_set_self_direct(slab,on) BIND(C,name="ghost_slab_set_self_direct") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT), VALUE :: on
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_exchange_self(slab,dir,nf,prune,fin,fout) BIND(C,name="ghost_slab_exchange_self") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT), VALUE :: dir, nf, prune
         TYPE(C_PTR) :: fin(*), fout(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_hd_front_z(slab,v,c,copy,prune,w) BIND(C,name="ghost_slab_hd_front_z") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         TYPE(C_PTR) :: v(3), c(3), w(6)
         INTEGER(C_INT), VALUE :: copy, prune
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_ypass(slab,sgn,nf,prune,fields) BIND(C,name="ghost_slab_ypass") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT), VALUE :: sgn, nf, prune
         TYPE(C_PTR) :: fields(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_slab_hd_back_z(slab,o,dt,nu,prune,w,v,c,f) BIND(C,name="ghost_slab_hd_back_z") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: slab
         INTEGER(C_INT), VALUE :: o, prune
         REAL(C_DOUBLE), VALUE :: dt, nu
         TYPE(C_PTR) :: w(3), v(3), c(3), f(3)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_set_tile_cfg(ctx,cfg) BIND(C,name="ghost_ctx_set_tile_cfg") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT), VALUE :: cfg
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_ctx_get_tile_cfg(ctx,cfg) BIND(C,name="ghost_ctx_get_tile_cfg") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT) :: cfg
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_hd_autotune(ctx,ord,dt,nu,vx,vy,vz,fx,fy,fz,cfg) BIND(C,name="ghost_hd_autotune") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, fx, fy, fz
         INTEGER(C_INT), VALUE :: ord
         REAL(C_DOUBLE), VALUE :: dt, nu
         INTEGER(C_INT) :: cfg
         INTEGER(C_INT) :: s
       END FUNCTION
       ! learned subgrid-stress closure (no GHOST counterpart)
       FUNCTION ghost_mlp_create(seed,mlp) BIND(C,name="ghost_mlp_create") RESULT(s)
         IMPORT :: C_INT, C_PTR
         INTEGER(C_INT), VALUE :: seed
         TYPE(C_PTR) :: mlp
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_mlp_destroy(mlp) BIND(C,name="ghost_mlp_destroy") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: mlp
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_mlp_set_stream(mlp,stream) BIND(C,name="ghost_mlp_set_stream") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: mlp, stream
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_mlp_get_params(mlp,params) BIND(C,name="ghost_mlp_get_params") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: mlp
         REAL(C_FLOAT) :: params(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_mlp_set_params(mlp,params) BIND(C,name="ghost_mlp_set_params") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: mlp
         REAL(C_FLOAT) :: params(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_mlp_forward(mlp,x,y,b) BIND(C,name="ghost_mlp_forward") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: mlp, x, y
         INTEGER(C_INT), VALUE :: b
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_mlp_gradients(mlp,x,t,b,grad,loss) BIND(C,name="ghost_mlp_gradients") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: mlp, x, t, grad
         INTEGER(C_INT), VALUE :: b
         REAL(C_DOUBLE) :: loss
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_mlp_train_step(mlp,x,t,b,lr,loss) BIND(C,name="ghost_mlp_train_step") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_FLOAT, C_DOUBLE
         TYPE(C_PTR), VALUE :: mlp, x, t
         INTEGER(C_INT), VALUE :: b
         REAL(C_FLOAT), VALUE :: lr
         REAL(C_DOUBLE) :: loss
         INTEGER(C_INT) :: s
       END FUNCTION
       ! large-eddy simulation: learned closure and GHOST's EDQNM eddy viscosity
       FUNCTION ghost_les_create(ctx,kc,les) BIND(C,name="ghost_les_create") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         INTEGER(C_INT), VALUE :: kc
         TYPE(C_PTR) :: les
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_destroy(les) BIND(C,name="ghost_les_destroy") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: les
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_truncate(les,fine,a,b) BIND(C,name="ghost_les_truncate") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: les, fine, a, b
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_samples(les,fine,vx,vy,vz,delta,x,tau) BIND(C,name="ghost_les_samples") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: les, fine, vx, vy, vz, x, tau
         REAL(C_FLOAT), VALUE :: delta
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_features(les,vx,vy,vz,gs,delta,x) BIND(C,name="ghost_les_features") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: les, vx, vy, vz, x
         REAL(C_FLOAT), VALUE :: gs, delta
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_spectral_features(les,e,x) BIND(C,name="ghost_les_spectral_features") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: les, e, x
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_tau_force(les,tau,ts,fx,fy,fz,ox,oy,oz) BIND(C,name="ghost_les_tau_force") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_FLOAT
         TYPE(C_PTR), VALUE :: les, tau, fx, fy, fz, ox, oy, oz
         REAL(C_FLOAT), VALUE :: ts
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_set_model(les,model,mlp,gs,ts,delta,kolmo) BIND(C,name="ghost_les_set_model") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: les, mlp
         INTEGER(C_INT), VALUE :: model
         REAL(C_DOUBLE), VALUE :: gs, ts, delta, kolmo
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_set_fallback(les,enable,blowup) BIND(C,name="ghost_les_set_fallback") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: les
         INTEGER(C_INT), VALUE :: enable
         REAL(C_DOUBLE), VALUE :: blowup
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_status(les,model,fell_back_at) BIND(C,name="ghost_les_status") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_LONG_LONG
         TYPE(C_PTR), VALUE :: les
         INTEGER(C_INT) :: model
         INTEGER(C_LONG_LONG) :: fell_back_at
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_set_time(les,t) BIND(C,name="ghost_les_set_time") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: les
         REAL(C_DOUBLE), VALUE :: t
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_closure_force(les,nu,vx,vy,vz,fx,fy,fz,ox,oy,oz) &
                BIND(C,name="ghost_les_closure_force") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: les, vx, vy, vz, fx, fy, fz, ox, oy, oz
         REAL(C_DOUBLE), VALUE :: nu
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_run(les,nsteps,ord,dt,nu,vx,vy,vz,fx,fy,fz) BIND(C,name="ghost_les_run") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: les, vx, vy, vz, fx, fy, fz
         INTEGER(C_INT), VALUE :: nsteps, ord
         REAL(C_DOUBLE), VALUE :: dt, nu
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_edqnm_last(les,tve,tepq,ek) BIND(C,name="ghost_les_edqnm_last") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: les
         REAL(C_DOUBLE) :: tve(*), tepq(*), ek(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_entrans(ctx,a,b,c,d,e,f,kin,ek) BIND(C,name="ghost_entrans") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: ek(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_heltrans(ctx,a,b,c,d,e,f,kin,hk) BIND(C,name="ghost_heltrans") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: hk(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_specpara(ctx,a,b,c,kin,hel,ek,hk) BIND(C,name="ghost_specpara") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         INTEGER(C_INT), VALUE :: kin, hel
         REAL(C_DOUBLE) :: ek(*), hk(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_specperp(ctx,a,b,c,kin,hel,ek,hk) BIND(C,name="ghost_specperp") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c
         INTEGER(C_INT), VALUE :: kin, hel
         REAL(C_DOUBLE) :: ek(*), hk(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_entpara(ctx,a,b,c,d,e,f,kin,ek) BIND(C,name="ghost_entpara") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: ek(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_entperp(ctx,a,b,c,d,e,f,kin,ek) BIND(C,name="ghost_entperp") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: ek(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_heltpara(ctx,a,b,c,d,e,f,kin,ek) BIND(C,name="ghost_heltpara") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: ek(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_heltperp(ctx,a,b,c,d,e,f,kin,ek) BIND(C,name="ghost_heltperp") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: ek(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_phaseshift(ctx,a,cre,cim) BIND(C,name="ghost_phaseshift") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a
         REAL(C_DOUBLE), VALUE :: cre, cim
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_forcing_slow(ctx,timef,fstep,fxold,fyold,fzold,fxnew,fynew,fznew,fx,fy,fz) &
                BIND(C,name="ghost_forcing_slow") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, fxold, fyold, fzold, fxnew, fynew, fznew, fx, fy, fz
         INTEGER(C_INT), VALUE :: timef, fstep
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_vector3(ctx,a,b,c,d,e,f,x,y,z) BIND(C,name="ghost_vector3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f, x, y, z
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_nonlin3(ctx,a,b,c,d,e,f,g,dir) BIND(C,name="ghost_nonlin3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b, c, d, e, f, g
         INTEGER(C_INT), VALUE :: dir
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_gauge3(ctx,a,b,c,g,dir) BIND(C,name="ghost_gauge3") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx, a, b, c, g
         INTEGER(C_INT), VALUE :: dir
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_mhd_run(ctx,nsteps,ord,dt,nu,mu,vx,vy,vz,ax,ay,az,fx,fy,fz,mx,my,mz) &
                BIND(C,name="ghost_mhd_run") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, ax, ay, az, fx, fy, fz, mx, my, mz
         INTEGER(C_INT), VALUE :: nsteps, ord
         REAL(C_DOUBLE), VALUE :: dt, nu, mu
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_phd_run(ctx,nsteps,ord,dt,nu,kappa,vx,vy,vz,th,fx,fy,fz,fs) &
                BIND(C,name="ghost_phd_run") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, vx, vy, vz, th, fx, fy, fz, fs
         INTEGER(C_INT), VALUE :: nsteps, ord
         REAL(C_DOUBLE), VALUE :: dt, nu, kappa
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_variance(ctx,a,kin,b) BIND(C,name="ghost_variance") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a
         INTEGER(C_INT), VALUE :: kin
         REAL(C_DOUBLE) :: b
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_spectrscc(ctx,a,shift,ek) BIND(C,name="ghost_spectrscc") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a
         REAL(C_DOUBLE), VALUE :: shift
         REAL(C_DOUBLE) :: ek(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_sctrans(ctx,a,b,isc,ek) BIND(C,name="ghost_sctrans") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, a, b
         INTEGER(C_INT), VALUE :: isc
         REAL(C_DOUBLE) :: ek(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_havgcomp(ctx,u,v,w,th,fo,bv,itype,gsh) BIND(C,name="ghost_havgcomp") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, u, v, w, th
         REAL(C_DOUBLE), VALUE :: fo, bv
         INTEGER(C_INT), VALUE :: itype
         REAL(C_DOUBLE) :: gsh(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_tbouss(ctx,u,v,w,th,fo,bv,avg,mx,mn) BIND(C,name="ghost_tbouss") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, u, v, w, th
         REAL(C_DOUBLE), VALUE :: fo, bv
         REAL(C_DOUBLE) :: avg(*), mx(*), mn(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_io_filename(dir,name,idx,width,buf,buflen) BIND(C,name="ghost_io_filename") RESULT(s)
         IMPORT :: C_INT, C_CHAR, C_SIZE_T
         CHARACTER(KIND=C_CHAR) :: dir(*), name(*), buf(*)
         INTEGER(C_INT), VALUE :: idx, width
         INTEGER(C_SIZE_T), VALUE :: buflen
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_io_write(ctx,var,path,swap) BIND(C,name="ghost_io_write") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_CHAR
         TYPE(C_PTR), VALUE :: ctx, var
         CHARACTER(KIND=C_CHAR) :: path(*)
         INTEGER(C_INT), VALUE :: swap
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_io_read(ctx,path,swap,var) BIND(C,name="ghost_io_read") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_CHAR
         TYPE(C_PTR), VALUE :: ctx, var
         CHARACTER(KIND=C_CHAR) :: path(*)
         INTEGER(C_INT), VALUE :: swap
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_io_output(ctx,spec,path,swap) BIND(C,name="ghost_io_output") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_CHAR
         TYPE(C_PTR), VALUE :: ctx, spec
         CHARACTER(KIND=C_CHAR) :: path(*)
         INTEGER(C_INT), VALUE :: swap
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_io_restart(ctx,path,swap,spec) BIND(C,name="ghost_io_restart") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_CHAR
         TYPE(C_PTR), VALUE :: ctx, spec
         CHARACTER(KIND=C_CHAR) :: path(*)
         INTEGER(C_INT), VALUE :: swap
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_evedqnm_hel(n,prec,kmax,kolmo,eold,hold,nu,time,hel,tepq,thpq,tve,tvh,ext,hxt) &
                BIND(C,name="ghost_evedqnm_hel") RESULT(s)
         IMPORT :: C_INT, C_DOUBLE
         INTEGER(C_INT), VALUE :: n, prec, hel
         REAL(C_DOUBLE), VALUE :: kmax, kolmo, nu, time
         REAL(C_DOUBLE) :: eold(*), hold(*), tepq(*), thpq(*), tve(*), tvh(*), ext(*), hxt(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_set_helicity(les,heli) BIND(C,name="ghost_les_set_helicity") RESULT(s)
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: les
         INTEGER(C_INT), VALUE :: heli
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_les_edqnm_last_hel(les,tvh,thpq,hk) BIND(C,name="ghost_les_edqnm_last_hel") RESULT(s)
         IMPORT :: C_INT, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: les
         REAL(C_DOUBLE) :: tvh(*), thpq(*), hk(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_evedqnm(n,prec,kmax,kolmo,eold,nu,time,tepq,tve,ext) BIND(C,name="ghost_evedqnm") RESULT(s)
         IMPORT :: C_INT, C_DOUBLE
         INTEGER(C_INT), VALUE :: n, prec
         REAL(C_DOUBLE), VALUE :: kmax, kolmo, nu, time
         REAL(C_DOUBLE) :: eold(*), tepq(*), tve(*), ext(*)
         INTEGER(C_INT) :: s
       END FUNCTION
       FUNCTION ghost_init_random_solenoidal(ctx,seed,kdn,kup,shape,amp,ox,oy,oz) &
                BIND(C,name="ghost_init_random_solenoidal") RESULT(s)
         IMPORT :: C_INT, C_INT32_T, C_PTR, C_DOUBLE
         TYPE(C_PTR), VALUE :: ctx, ox, oy, oz
         INTEGER(C_INT32_T) :: seed
         REAL(C_DOUBLE), VALUE :: kdn, kup, amp
         INTEGER(C_INT), VALUE :: shape
         INTEGER(C_INT) :: s
       END FUNCTION
      END INTERFACE

      CONTAINS

      ! Creates the run's context; call once after nx,ny,nz and the box are
      ! known (main3D.fpp:1721).  Stops on failure, like GHOST's setup.
      SUBROUTINE ghost_gpu_init(nx,ny,nz,Lx,Ly,Lz,arbsize,gpkind)
      INTEGER, INTENT(IN) :: nx, ny, nz, arbsize, gpkind
      DOUBLE PRECISION, INTENT(IN) :: Lx, Ly, Lz
      CALL ghost_gpu_check(ghost_ctx_create(nx,ny,nz,Lx,Ly,Lz,arbsize,gpkind,gctx), &
                           'ghost_ctx_create')
      END SUBROUTINE ghost_gpu_init

      SUBROUTINE ghost_gpu_check(s,where)
      INTEGER(C_INT), INTENT(IN) :: s
      CHARACTER(len=*), INTENT(IN) :: where
      CHARACTER(kind=C_CHAR), POINTER :: msg(:)
      INTEGER :: n
      IF (s.ne.GHOST_OK) THEN
         CALL C_F_POINTER(ghost_last_error_string(), msg, [1024])
         n = 0
         DO WHILE (n.lt.1024)
            IF (msg(n+1).eq.C_NULL_CHAR) EXIT
            n = n+1
         END DO
         PRINT *, where, ': status ', s, ': ', msg(1:n)
         STOP
      ENDIF
      END SUBROUTINE ghost_gpu_check

      END MODULE ghost_gpu

!=================================================================
! Drop-in replacements with GHOST's interfaces.  They take GHOST's
! module state (grid, mpivars) for the array shapes; the plan handle
! travels in FFTPLAN%planr of the fftplans module.
!=================================================================
      SUBROUTINE fftp3d_create_plan(plan,n,fftdir,flags)
      USE fftplans
      USE ghost_gpu
      IMPLICIT NONE
      TYPE(FFTPLAN), INTENT(OUT) :: plan
      INTEGER, INTENT(IN) :: n(3), fftdir, flags
      TYPE(C_PTR) :: p
      INTEGER(C_INT) :: nn(3)
      nn = n
      CALL ghost_gpu_check(ghost_fftp3d_create_plan(gctx,nn,fftdir,flags,p), &
                           'fftp3d_create_plan')
      plan%planr = TRANSFER(p,plan%planr)
      plan%nx = n(1)
      plan%ny = n(2)
      plan%nz = n(3)
      END SUBROUTINE fftp3d_create_plan

      SUBROUTINE fftp3d_destroy_plan(plan)
      USE fftplans
      USE ghost_gpu
      IMPLICIT NONE
      TYPE(FFTPLAN), INTENT(INOUT) :: plan
      CALL ghost_gpu_check(ghost_fftp3d_destroy_plan(TRANSFER(plan%planr,C_NULL_PTR)), &
                           'fftp3d_destroy_plan')
      END SUBROUTINE fftp3d_destroy_plan

      SUBROUTINE fftp3d_real_to_complex(plan,in,out,comm)
      USE fprecision
      USE fftplans
      USE ghost_gpu
      IMPLICIT NONE
      TYPE(FFTPLAN), INTENT(IN) :: plan
      REAL(KIND=GP), INTENT(IN), TARGET :: in(plan%nx,plan%ny,plan%nz)
      COMPLEX(KIND=GP), INTENT(OUT), TARGET :: out(plan%nz,plan%ny,plan%nx/2+1)
      INTEGER, INTENT(IN) :: comm
      CALL ghost_gpu_check(ghost_fftp3d_real_to_complex(TRANSFER(plan%planr,C_NULL_PTR), &
                           C_LOC(in),C_LOC(out)),'fftp3d_real_to_complex')
      END SUBROUTINE fftp3d_real_to_complex

      SUBROUTINE fftp3d_complex_to_real(plan,in,out,comm)
      USE fprecision
      USE fftplans
      USE ghost_gpu
      IMPLICIT NONE
      TYPE(FFTPLAN), INTENT(IN) :: plan
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: in(plan%nz,plan%ny,plan%nx/2+1)
      REAL(KIND=GP), INTENT(OUT), TARGET :: out(plan%nx,plan%ny,plan%nz)
      INTEGER, INTENT(IN) :: comm
      CALL ghost_gpu_check(ghost_fftp3d_complex_to_real(TRANSFER(plan%planr,C_NULL_PTR), &
                           C_LOC(in),C_LOC(out)),'fftp3d_complex_to_real')
      END SUBROUTINE fftp3d_complex_to_real

      SUBROUTINE derivk3(a,b,dir)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1)
      COMPLEX(KIND=GP), INTENT(OUT), TARGET :: b(nz,ny,nx/2+1)
      INTEGER, INTENT(IN) :: dir
      CALL ghost_gpu_check(ghost_derivk3(gctx,C_LOC(a),C_LOC(b),dir),'derivk3')
      END SUBROUTINE derivk3

      SUBROUTINE laplak3(a,b)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1)
      COMPLEX(KIND=GP), INTENT(OUT), TARGET :: b(nz,ny,nx/2+1)
      CALL ghost_gpu_check(ghost_laplak3(gctx,C_LOC(a),C_LOC(b)),'laplak3')
      END SUBROUTINE laplak3

      SUBROUTINE rotor3(a,b,c,dir)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1), b(nz,ny,nx/2+1)
      COMPLEX(KIND=GP), INTENT(OUT), TARGET :: c(nz,ny,nx/2+1)
      INTEGER, INTENT(IN) :: dir
      CALL ghost_gpu_check(ghost_rotor3(gctx,C_LOC(a),C_LOC(b),C_LOC(c),dir),'rotor3')
      END SUBROUTINE rotor3

      SUBROUTINE prodre3(a,b,c,d,e,f)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1), b(nz,ny,nx/2+1), c(nz,ny,nx/2+1)
      COMPLEX(KIND=GP), INTENT(OUT), TARGET :: d(nz,ny,nx/2+1), e(nz,ny,nx/2+1), f(nz,ny,nx/2+1)
      CALL ghost_gpu_check(ghost_prodre3(gctx,C_LOC(a),C_LOC(b),C_LOC(c), &
                           C_LOC(d),C_LOC(e),C_LOC(f)),'prodre3')
      END SUBROUTINE prodre3

      SUBROUTINE nonlhd3(a,b,c,g,dir)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1), b(nz,ny,nx/2+1), c(nz,ny,nx/2+1)
      COMPLEX(KIND=GP), INTENT(OUT), TARGET :: g(nz,ny,nx/2+1)
      INTEGER, INTENT(IN) :: dir
      CALL ghost_gpu_check(ghost_nonlhd3(gctx,C_LOC(a),C_LOC(b),C_LOC(c),C_LOC(g),dir), &
                           'nonlhd3')
      END SUBROUTINE nonlhd3

      SUBROUTINE energy(a,b,c,d,kin)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1), b(nz,ny,nx/2+1), c(nz,ny,nx/2+1)
      DOUBLE PRECISION, INTENT(OUT) :: d
      INTEGER, INTENT(IN) :: kin
      REAL(C_DOUBLE) :: dd
      CALL ghost_gpu_check(ghost_energy(gctx,C_LOC(a),C_LOC(b),C_LOC(c),dd,kin),'energy')
      d = dd
      END SUBROUTINE energy

      SUBROUTINE helicity(a,b,c,d)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1), b(nz,ny,nx/2+1), c(nz,ny,nx/2+1)
      DOUBLE PRECISION, INTENT(OUT) :: d
      REAL(C_DOUBLE) :: dd
      CALL ghost_gpu_check(ghost_helicity(gctx,C_LOC(a),C_LOC(b),C_LOC(c),dd),'helicity')
      d = dd
      END SUBROUTINE helicity

      SUBROUTINE cross(a,b,c,d,e,f,g,kin)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1), b(nz,ny,nx/2+1), c(nz,ny,nx/2+1)
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: d(nz,ny,nx/2+1), e(nz,ny,nx/2+1), f(nz,ny,nx/2+1)
      DOUBLE PRECISION, INTENT(OUT) :: g
      INTEGER, INTENT(IN) :: kin
      REAL(C_DOUBLE) :: gg
      CALL ghost_gpu_check(ghost_cross(gctx,C_LOC(a),C_LOC(b),C_LOC(c),C_LOC(d), &
                           C_LOC(e),C_LOC(f),gg,kin),'cross')
      g = gg
      END SUBROUTINE cross

      SUBROUTINE maxabs(a,b,c,d,kin)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1), b(nz,ny,nx/2+1), c(nz,ny,nx/2+1)
      REAL(KIND=GP), INTENT(OUT) :: d
      INTEGER, INTENT(IN) :: kin
      REAL(C_DOUBLE) :: dd
      CALL ghost_gpu_check(ghost_maxabs(gctx,C_LOC(a),C_LOC(b),C_LOC(c),dd,kin),'maxabs')
      d = REAL(dd,KIND=GP)
      END SUBROUTINE maxabs

      SUBROUTINE spectrumc(a,b,c,kin,hel,Ektot,Hktot)
      USE fprecision
      USE grid
      USE kes
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET :: a(nz,ny,nx/2+1), b(nz,ny,nx/2+1), c(nz,ny,nx/2+1)
      INTEGER, INTENT(IN) :: kin, hel
      DOUBLE PRECISION, INTENT(OUT), DIMENSION(nmax/2+1) :: Ektot, Hktot
      CALL ghost_gpu_check(ghost_spectrumc(gctx,C_LOC(a),C_LOC(b),C_LOC(c),kin,hel, &
                           Ektot,Hktot),'spectrumc')
      END SUBROUTINE spectrumc

!-----------------------------------------------------------------
! io_write / io_read (mpiio/binary_io.f90:13-186) for a single-rank
! run (ksta = 1, kend = nz): the file name is GHOST's mangled
! dir/fname.nmb.out; reads byte-swap when iswap > 0, as GHOST's do.
!-----------------------------------------------------------------
      SUBROUTINE io_write(unit,dir,fname,nmb,plan,var)
      USE fprecision
      USE iovar
      USE ghost_gpu
      IMPLICIT NONE
      TYPE(IOPLAN), INTENT(IN) :: plan
      REAL(KIND=GP), INTENT(INOUT), TARGET :: var(plan%nx,plan%ny,plan%ksta:plan%kend)
      INTEGER, INTENT(IN) :: unit
      CHARACTER(len=100), INTENT(IN) :: dir
      CHARACTER(len=*), INTENT(IN) :: nmb
      CHARACTER(len=*), INTENT(IN) :: fname
      CALL ghost_gpu_check(ghost_io_write(gctx,C_LOC(var), &
           trim(dir)//'/'//fname//'.'//nmb//'.out'//C_NULL_CHAR,0),'io_write')
      END SUBROUTINE io_write

      SUBROUTINE io_read(unit,dir,fname,nmb,plan,var)
      USE fprecision
      USE iovar
      USE ghost_gpu
      IMPLICIT NONE
      TYPE(IOPLAN), INTENT(IN) :: plan
      REAL(KIND=GP), INTENT(OUT), TARGET :: var(plan%nx,plan%ny,plan%ksta:plan%kend)
      INTEGER, INTENT(IN) :: unit
      CHARACTER(len=100), INTENT(IN) :: dir
      CHARACTER(len=*), INTENT(IN) :: nmb
      CHARACTER(len=*), INTENT(IN) :: fname
      INTEGER(C_INT) :: swap
      swap = 0
      IF (iswap.gt.0) swap = 1
      CALL ghost_gpu_check(ghost_io_read(gctx, &
           trim(dir)//'/'//fname//'.'//nmb//'.out'//C_NULL_CHAR,swap,C_LOC(var)),'io_read')
      END SUBROUTINE io_read

!-----------------------------------------------------------------
! entrans / heltrans (pseudospec3D_hd.f90:1629-1949): the shell sums
! on the device, GHOST's text file (Dkk*k, sum/Dkk) written here.
!-----------------------------------------------------------------
      SUBROUTINE entrans(a,b,c,d,e,f,nmb,kin)
      USE fprecision
      USE grid
      USE kes
      USE boxsize
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET, DIMENSION(nz,ny,nx/2+1) :: a,b,c,d,e,f
      INTEGER, INTENT(IN) :: kin
      CHARACTER(len=*), INTENT(IN) :: nmb
      DOUBLE PRECISION, DIMENSION(nmax/2+1) :: Ektot
      INTEGER :: i
      CALL ghost_gpu_check(ghost_entrans(gctx,C_LOC(a),C_LOC(b),C_LOC(c),C_LOC(d),C_LOC(e), &
                           C_LOC(f),kin,Ektot),'entrans')
      IF (kin.eq.0) THEN
         OPEN(1,file='mtransfer.' // nmb // '.txt')
      ELSEIF (kin.eq.1) THEN
         OPEN(1,file='ktransfer.' // nmb // '.txt')
      ELSEIF (kin.eq.2) THEN
         OPEN(1,file='jtransfer.' // nmb // '.txt')
      ELSEIF (kin.eq.3) THEN
         OPEN(1,file='mcrostran.' // nmb // '.txt')
      ELSE
         OPEN(1,file='kcrostran.' // nmb // '.txt')
      ENDIF
      DO i = 1,nmax/2+1
         WRITE(1,FMT='(E13.6,E23.15)') Dkk*i,Ektot(i)/Dkk
      END DO
      CLOSE(1)
      END SUBROUTINE entrans

      SUBROUTINE heltrans(a,b,c,d,e,f,nmb,kin)
      USE fprecision
      USE grid
      USE kes
      USE boxsize
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET, DIMENSION(nz,ny,nx/2+1) :: a,b,c,d,e,f
      INTEGER, INTENT(IN) :: kin
      CHARACTER(len=*), INTENT(IN) :: nmb
      DOUBLE PRECISION, DIMENSION(nmax/2+1) :: Hktot
      INTEGER :: i
      CALL ghost_gpu_check(ghost_heltrans(gctx,C_LOC(a),C_LOC(b),C_LOC(c),C_LOC(d),C_LOC(e), &
                           C_LOC(f),kin,Hktot),'heltrans')
      IF (kin.eq.0) THEN
         OPEN(1,file='hmtransfer.' // nmb // '.txt')
      ELSE
         OPEN(1,file='hktransfer.' // nmb // '.txt')
      ENDIF
      DO i = 1,nmax/2+1
         WRITE(1,FMT='(E13.6,E23.15)') Dkk*i,Hktot(i)/Dkk
      END DO
      CLOSE(1)
      END SUBROUTINE heltrans

!-----------------------------------------------------------------
! tbouss (pseudospec3D_bouss.f90:611-711): the profiles on the device,
! GHOST's three appended text files written here.
!-----------------------------------------------------------------
      SUBROUTINE tbouss(u, v, w, s, t, dt, fo, bv)
      USE fprecision
      USE grid
      USE ghost_gpu
      IMPLICIT NONE
      COMPLEX(KIND=GP), INTENT(IN), TARGET, DIMENSION(nz,ny,nx/2+1) :: u,v,w,s
      REAL(KIND=GP), INTENT(IN) :: dt, fo, bv
      INTEGER, INTENT(IN) :: t
      DOUBLE PRECISION :: gxavg(11),gxmax(11),gxmin(11)
      CALL ghost_gpu_check(ghost_tbouss(gctx,C_LOC(u),C_LOC(v),C_LOC(w),C_LOC(s), &
           DBLE(fo),DBLE(bv),gxavg,gxmax,gxmin),'tbouss')
      OPEN(1,file='tboussavg.txt',position='append')
      WRITE(1,20) (t-1)*dt,gxavg
      CLOSE(1)
      OPEN(1,file='tboussmax.txt',position='append')
      WRITE(1,20) (t-1)*dt,gxmax
      CLOSE(1)
      OPEN(1,file='tboussmin.txt',position='append')
      WRITE(1,20) (t-1)*dt,gxmin
      CLOSE(1)
   20 FORMAT( E13.6,1x,11(E26.18,1x) )
      END SUBROUTINE tbouss
