!##############################################################################
!
! ash3d_b200_shim.f90 -- ISO_C_BINDING drop-in for Ash3d's transport path.
!
! Build Ash3d with USEPOINTERS=T (src/makefile:80) so that c_loc() of the
! module arrays is legal, compile this file in place of
!   src/AdvectionHorz.f90, src/AdvectionHorz_DCU.f90,
!   src/AdvectionVert_DCU.f90, src/Diffusion.F90, src/Set_BC.f90,
!   src/Adjust_dt.f90, src/TimeStepTotals.f90
! and link libash3d_b200.so.  Ash3d.F90 keeps calling the same names with the
! same arguments:
!   Set_BC(bc_code)            src/Set_BC.f90:15
!   AdvectHorz(itoggle)        src/AdvectionHorz.f90:47
!   AdvectVert                 src/AdvectionVert_DCU.f90:64
!   DiffuseHorz(i), DiffuseVert  src/Diffusion.F90:151,232
!   Adjust_DT(mesostep)        src/Adjust_dt.f90:19
!   TimeStepTotals(itime)      src/TimeStepTotals.f90:17
! A nonzero status from the library is reported on errlog and ends the run
! with "stop 1", the reference's error convention (e.g. src/Set_BC.f90:119-123).
!
! The concentration lives on the GPU between calls.  B200_Download copies it
! back into concen_pd(:,:,:,:,ts0) (and the outflow/deposit arrays) before
! the host reads them: before Gen_Output_Vars/output_results and restart
! writes.  B200_Upload sends a host-modified field back (restart loads).
! This file is written against the reference's module interfaces and is not
! compiled in this repository's test suite (no Fortran compiler in the image).
!##############################################################################

      module B200_Transport

      use iso_c_binding

      implicit none

      private
      public B200_Init, B200_Finalize, B200_Upload, B200_Download, B200_Check, &
             B200_StepPrologue, B200_AddSource, B200_SetWinds, B200_SetMetSteps, &
             B200_InterpWinds, B200_SetTopo, B200_SetUmbrella, B200_AddUmbrellaWinds, &
             B200_AddSourceUmbrella, B200_OutputAshcon, B200_RestartLoad, b200_ctx

      type, bind(C) :: a3g_grid_desc
        integer(c_int32_t) :: nx, ny, nz, ns
        integer(c_int32_t) :: periodic, latlon
        real(c_double)     :: dx, dy
      end type a3g_grid_desc

      type, bind(C) :: a3g_params
        integer(c_int32_t) :: limiter, use_cn, use_diffusion, fast_subgrid, nocycle, zscaling_id
        real(c_double)     :: cfl, dt_min, dt_max, imp_fac, imp_dt_fac, eps_thresh, eps_small
        real(c_double)     :: cloudcon_grid_thresh, magma_density
      end type a3g_params

      type(c_ptr), save :: b200_ctx = c_null_ptr

      interface
        subroutine a3g_default_params(p) bind(C, name="a3g_default_params")
          import :: a3g_params
          type(a3g_params), intent(out) :: p
        end subroutine
        function a3g_last_error() bind(C, name="a3g_last_error") result(msg)
          import :: c_ptr
          type(c_ptr) :: msg
        end function
        integer(c_int) function a3g_create(grid, prm, device, ctx) bind(C, name="a3g_create")
          import :: a3g_grid_desc, a3g_params, c_int, c_ptr
          type(a3g_grid_desc), intent(in) :: grid
          type(a3g_params), intent(in) :: prm
          integer(c_int), value :: device
          type(c_ptr), intent(out) :: ctx
        end function
        integer(c_int) function a3g_destroy(ctx) bind(C, name="a3g_destroy")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
        end function
        integer(c_int) function a3g_set_geometry(ctx, kap, snx, sny, snz, dz) bind(C, name="a3g_set_geometry")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, kap, snx, sny, snz, dz
        end function
        integer(c_int) function a3g_set_diffusivity(ctx, kx, ky, kz) bind(C, name="a3g_set_diffusivity")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, kx, ky, kz
        end function
        integer(c_int) function a3g_set_fall_velocity(ctx, vf) bind(C, name="a3g_set_fall_velocity")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, vf
        end function
        integer(c_int) function a3g_set_aloft(ctx, aloft) bind(C, name="a3g_set_aloft")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, aloft
        end function
        integer(c_int) function a3g_set_winds(ctx, vx, vy, vz) bind(C, name="a3g_set_winds")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, vx, vy, vz
        end function
        integer(c_int) function a3g_set_met_steps(ctx, xl, yl, zl, xn, yn, zn) bind(C, name="a3g_set_met_steps")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, xl, yl, zl, xn, yn, zn
        end function
        integer(c_int) function a3g_interp_winds(ctx, frac) bind(C, name="a3g_interp_winds")
          import :: c_int, c_ptr, c_double
          type(c_ptr), value :: ctx
          real(c_double), value :: frac
        end function
        integer(c_int) function a3g_set_umbrella(ctx, iv, jv, ib, it, sten) bind(C, name="a3g_set_umbrella")
          import :: c_int, c_ptr, c_int32_t
          type(c_ptr), value :: ctx, sten
          integer(c_int32_t), value :: iv, jv, ib, it
        end function
        integer(c_int) function a3g_add_umbrella_winds(ctx, i0, i1, j0, j1, ux, uy) &
            bind(C, name="a3g_add_umbrella_winds")
          import :: c_int, c_ptr, c_int32_t
          type(c_ptr), value :: ctx, ux, uy
          integer(c_int32_t), value :: i0, i1, j0, j1
        end function
        integer(c_int) function a3g_add_source_umbrella(ctx, flux, dt) bind(C, name="a3g_add_source_umbrella")
          import :: c_int, c_ptr, c_double
          type(c_ptr), value :: ctx, flux
          real(c_double), value :: dt
        end function
        integer(c_int) function a3g_set_topo(ctx, dhdx, dhdy, ddx, ddy, scc, ztop) bind(C, name="a3g_set_topo")
          import :: c_int, c_ptr, c_double
          type(c_ptr), value :: ctx, dhdx, dhdy, ddx, ddy, scc
          real(c_double), value :: ztop
        end function
        integer(c_int) function a3g_upload_concen(ctx, c) bind(C, name="a3g_upload_concen")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, c
        end function
        integer(c_int) function a3g_download_concen(ctx, c) bind(C, name="a3g_download_concen")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, c
        end function
        integer(c_int) function a3g_upload_outflow(ctx, a, b, c, d, e, f) bind(C, name="a3g_upload_outflow")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, a, b, c, d, e, f
        end function
        integer(c_int) function a3g_download_outflow(ctx, a, b, c, d, e, f, dep) &
            bind(C, name="a3g_download_outflow")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, a, b, c, d, e, f, dep
        end function
        integer(c_int) function a3g_output_ashcon(ctx, ash, dep) bind(C, name="a3g_output_ashcon")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, ash, dep
        end function
        integer(c_int) function a3g_restart_load(ctx, ash, dep) bind(C, name="a3g_restart_load")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, ash, dep
        end function
        integer(c_int) function a3g_step_prologue(ctx) bind(C, name="a3g_step_prologue")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
        end function
        integer(c_int) function a3g_set_dt(ctx, dt) bind(C, name="a3g_set_dt")
          import :: c_int, c_ptr, c_double
          type(c_ptr), value :: ctx
          real(c_double), value :: dt
        end function
        integer(c_int) function a3g_add_source_column(ctx, iv, jv, flux, dt) bind(C, name="a3g_add_source_column")
          import :: c_int, c_int32_t, c_ptr, c_double
          type(c_ptr), value :: ctx, flux
          integer(c_int32_t), value :: iv, jv
          real(c_double), value :: dt
        end function
        integer(c_int) function a3g_set_bc(ctx, code) bind(C, name="a3g_set_bc")
          import :: c_int, c_int32_t, c_ptr
          type(c_ptr), value :: ctx
          integer(c_int32_t), value :: code
        end function
        integer(c_int) function a3g_advect_horz(ctx, itoggle, iv, jv, kv) bind(C, name="a3g_advect_horz")
          import :: c_int, c_int32_t, c_ptr
          type(c_ptr), value :: ctx
          integer(c_int32_t), value :: itoggle, iv, jv, kv
        end function
        integer(c_int) function a3g_advect_vert(ctx) bind(C, name="a3g_advect_vert")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
        end function
        integer(c_int) function a3g_diffuse_horz(ctx, itime) bind(C, name="a3g_diffuse_horz")
          import :: c_int, c_int32_t, c_ptr
          type(c_ptr), value :: ctx
          integer(c_int32_t), value :: itime
        end function
        integer(c_int) function a3g_diffuse_vert(ctx) bind(C, name="a3g_diffuse_vert")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
        end function
        integer(c_int) function a3g_adjust_dt(ctx, time, nwt, simtime, dt) bind(C, name="a3g_adjust_dt")
          import :: c_int, c_ptr, c_double
          type(c_ptr), value :: ctx
          real(c_double), value :: time, nwt, simtime
          real(c_double), intent(out) :: dt
        end function
        integer(c_int) function a3g_set_fall_velocity_meso(ctx, vf, per_grain) &
            bind(C, name="a3g_set_fall_velocity_meso")
          import :: c_int, c_ptr, c_int32_t
          type(c_ptr), value :: ctx, vf
          integer(c_int32_t), value :: per_grain
        end function
        integer(c_int) function a3g_adjust_dt_meso(ctx, slot, shift, time, nwt, simtime, dt) &
            bind(C, name="a3g_adjust_dt_meso")
          import :: c_int, c_ptr, c_int32_t, c_double
          type(c_ptr), value :: ctx
          integer(c_int32_t), value :: slot, shift
          real(c_double), value :: time, nwt, simtime
          real(c_double), intent(out) :: dt
        end function
        integer(c_int) function a3g_timestep_totals(ctx, out4, mass) bind(C, name="a3g_timestep_totals")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, out4, mass
        end function
        integer(c_int) function a3g_get_subgrid(ctx, box) bind(C, name="a3g_get_subgrid")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, box
        end function
      end interface

      contains

      !------------------------------------------------------------------------
      ! Maps a nonzero library status to the reference's errlog + stop 1.
      subroutine B200_Check(rc, where)
        use io_units
        integer(c_int), intent(in) :: rc
        character(len=*), intent(in) :: where
        character(kind=c_char), pointer :: msg(:)
        integer :: n
        if (rc .eq. 0) return
        call c_f_pointer(a3g_last_error(), msg, [512])
        n = 0
        do while (n .lt. 512)
          if (msg(n+1) .eq. c_null_char) exit
          n = n + 1
        enddo
        do io=1,2;if(VB(io).le.verbosity_error)then
          write(errlog(io),*)"ERROR (B200) in ", where, ": status ", rc, " ", msg(1:n)
        endif;enddo
        stop 1
      end subroutine B200_Check

      !------------------------------------------------------------------------
      ! After alloc_arrays, calc_mesh_params, Get_Topo, calc_s_mesh (so that the
      ! ZScaling_ID 2 geometry is the scaled one) and Allocate_Diff
      ! (src/Ash3d.F90:230-240).
      subroutine B200_Init(device)
        use global_param, only : CFL, DT_MIN, DT_MAX, useDiffusion, useCN, EPS_THRESH, EPS_SMALL
        use mesh,         only : nxmax, nymax, nzmax, nsmax, IsPeriodic, IsLatLon, dx, dy, &
                                 kappa_pd, sigma_nx_pd, sigma_ny_pd, sigma_nz_pd, dz_vec_pd, ZScaling_ID
        use solution,     only : vf_pd
        use Diffusion,    only : kx, ky, kz, Imp_fac, Imp_DT_fac
        use Output_Vars,  only : CLOUDCON_GRID_THRESH
        use Tephra,       only : MagmaDensity
        integer, intent(in) :: device
        type(a3g_grid_desc) :: g
        type(a3g_params) :: p
        g%nx = nxmax; g%ny = nymax; g%nz = nzmax; g%ns = nsmax
        g%periodic = merge(1, 0, IsPeriodic); g%latlon = merge(1, 0, IsLatLon)
        g%dx = dx; g%dy = dy
        call a3g_default_params(p)
        p%use_cn = merge(1, 0, useCN)
        p%use_diffusion = merge(1, 0, useDiffusion)
#ifdef FAST_SUBGRID
        p%fast_subgrid = 1
#endif
        p%zscaling_id = ZScaling_ID
        p%cfl = CFL; p%dt_min = DT_MIN; p%dt_max = DT_MAX
        p%imp_fac = Imp_fac; p%imp_dt_fac = Imp_DT_fac; p%eps_thresh = EPS_THRESH
        p%eps_small = EPS_SMALL; p%cloudcon_grid_thresh = CLOUDCON_GRID_THRESH
        p%magma_density = MagmaDensity
        call B200_Check(a3g_create(g, p, int(device, c_int), b200_ctx), "a3g_create")
        call B200_Check(a3g_set_geometry(b200_ctx, c_loc(kappa_pd), c_loc(sigma_nx_pd), &
                        c_loc(sigma_ny_pd), c_loc(sigma_nz_pd), c_loc(dz_vec_pd)), "a3g_set_geometry")
        call B200_Check(a3g_set_diffusivity(b200_ctx, c_loc(kx), c_loc(ky), c_loc(kz)), "a3g_set_diffusivity")
        call B200_Check(a3g_set_fall_velocity(b200_ctx, c_loc(vf_pd)), "a3g_set_fall_velocity")
      end subroutine B200_Init

      subroutine B200_Finalize
        integer(c_int) :: rc
        rc = a3g_destroy(b200_ctx)
        b200_ctx = c_null_ptr
      end subroutine B200_Finalize

      ! concen_pd(:,:,:,:,ts0) and the outflow accumulators -> device
      subroutine B200_Upload
        use mesh,     only : ts0
        use solution, only : concen_pd, outflow_yz1_pd, outflow_yz2_pd, outflow_xz1_pd, &
                             outflow_xz2_pd, outflow_xy1_pd, outflow_xy2_pd
        call B200_Check(a3g_upload_concen(b200_ctx, c_loc(concen_pd(-1,-1,-1,1,ts0))), "a3g_upload_concen")
        call B200_Check(a3g_upload_outflow(b200_ctx, c_loc(outflow_yz1_pd), c_loc(outflow_yz2_pd), &
                        c_loc(outflow_xz1_pd), c_loc(outflow_xz2_pd), c_loc(outflow_xy1_pd), &
                        c_loc(outflow_xy2_pd)), "a3g_upload_outflow")
      end subroutine B200_Upload

      ! device -> concen_pd(ts0) and ts1 (the state after the step), outflows, deposit
      subroutine B200_Download
        use mesh,     only : ts0, ts1
        use solution, only : concen_pd, outflow_yz1_pd, outflow_yz2_pd, outflow_xz1_pd, &
                             outflow_xz2_pd, outflow_xy1_pd, outflow_xy2_pd, DepositGranularity
        call B200_Check(a3g_download_concen(b200_ctx, c_loc(concen_pd(-1,-1,-1,1,ts1))), "a3g_download_concen")
        concen_pd(:,:,:,:,ts0) = concen_pd(:,:,:,:,ts1)
        call B200_Check(a3g_download_outflow(b200_ctx, c_loc(outflow_yz1_pd), c_loc(outflow_yz2_pd), &
                        c_loc(outflow_xz1_pd), c_loc(outflow_xz2_pd), c_loc(outflow_xy1_pd), &
                        c_loc(outflow_xy2_pd), c_loc(DepositGranularity)), "a3g_download_outflow")
      end subroutine B200_Download

      ! replaces the two full-array copies of src/Ash3d.F90:376-378
      subroutine B200_StepPrologue
        call B200_Check(a3g_step_prologue(b200_ctx), "a3g_step_prologue")
      end subroutine B200_StepPrologue

      ! replaces the vent-column update of src/Ash3d.F90:428-431
      subroutine B200_AddSource
        use mesh,      only : ivent, jvent
        use Source,    only : SourceNodeFlux
        use time_data, only : dt
        call B200_Check(a3g_add_source_column(b200_ctx, int(ivent, c_int32_t), int(jvent, c_int32_t), &
                        c_loc(SourceNodeFlux), real(dt, c_double)), "a3g_add_source_column")
      end subroutine B200_AddSource

      ! host-interpolated FP64 winds (MesoInterpolater left unchanged)
      subroutine B200_SetWinds
        use solution, only : vx_pd, vy_pd, vz_pd
        call B200_Check(a3g_set_winds(b200_ctx, c_loc(vx_pd), c_loc(vy_pd), c_loc(vz_pd)), "a3g_set_winds")
      end subroutine B200_SetWinds

      ! device interpolation: upload the bracketing FP32 met steps once per met
      ! step, right after each call of Read_NextMesoStep in MesoInterpolater
      ! (src/MesoInterpolater.f90:142 and :189), so that FAST_DT's
      ! Adjust_DT(.true.) that follows it reads them on the device.  The met
      ! steps' fall velocities go with them: per cell when a fall model fills
      ! vf_meso_next_step_sp (useCalcFallVel), else the input file's
      ! real(Tephra_v_s, sp), which Read_NextMesoStep puts in every cell
      ! (:567-574).
      subroutine B200_SetMetSteps
        use global_param, only : useCalcFallVel
        use mesh,      only : nsmax
        use Tephra,    only : Tephra_v_s
        use wind_grid, only : vx_meso_last_step_sp, vy_meso_last_step_sp, vz_meso_last_step_sp, &
                              vx_meso_next_step_sp, vy_meso_next_step_sp, vz_meso_next_step_sp, &
                              vf_meso_next_step_sp
        real(c_float), allocatable, target :: vs(:)
        call B200_Check(a3g_set_met_steps(b200_ctx, c_loc(vx_meso_last_step_sp), c_loc(vy_meso_last_step_sp), &
                        c_loc(vz_meso_last_step_sp), c_loc(vx_meso_next_step_sp), &
                        c_loc(vy_meso_next_step_sp), c_loc(vz_meso_next_step_sp)), "a3g_set_met_steps")
        if (useCalcFallVel) then
          call B200_Check(a3g_set_fall_velocity_meso(b200_ctx, c_loc(vf_meso_next_step_sp), 0_c_int32_t), &
                          "a3g_set_fall_velocity_meso")
        else
          allocate(vs(nsmax))
          vs = real(Tephra_v_s(1:nsmax), c_float)
          call B200_Check(a3g_set_fall_velocity_meso(b200_ctx, c_loc(vs), 1_c_int32_t), &
                          "a3g_set_fall_velocity_meso")
          deallocate(vs)
        endif
      end subroutine B200_SetMetSteps

      ! ... and interpolate on the device every step (src/MesoInterpolater.f90:207-223)
      subroutine B200_InterpWinds(frac)
        real(kind=8), intent(in) :: frac
        call B200_Check(a3g_interp_winds(b200_ctx, real(frac, c_double)), "a3g_interp_winds")
      end subroutine B200_InterpWinds

      ! useTopo: bind the terrain terms once, after Get_Topo and calc_s_mesh
      ! (src/Ash3d.F90:233-240).  vh is then formed on the device after every
      ! B200_SetWinds / B200_InterpWinds, in place of Calc_Vmod_Topo
      ! (src/Ash3d.F90:398).  dhdx_comp and dhdy_comp are private to module
      ! Topography (src/Topography.f90:181-182) and need the public attribute.
      subroutine B200_SetTopo
        use mesh,       only : s_cc_pd, Ztop
        use Topography, only : dhdx_comp, dhdy_comp, DelDxonD_cc, DelDyonD_cc
        call B200_Check(a3g_set_topo(b200_ctx, c_loc(dhdx_comp), c_loc(dhdy_comp), c_loc(DelDxonD_cc), &
                        c_loc(DelDyonD_cc), c_loc(s_cc_pd), real(Ztop, c_double)), "a3g_set_topo")
      end subroutine B200_SetTopo

      ! Umbrella source: once, after Allocate_Source_Umbrella (src/Ash3d.F90:242-244).
      ! AvgStenc_Umbrella is private to module Source_Umbrella, so the stencil is
      ! formed here from kappa_pd exactly as src/Source_Umbrella.f90:127-138 does.
      subroutine B200_SetUmbrella
        use mesh,            only : nzmax, kappa_pd, ivent, jvent
        use Source_Umbrella, only : ibase, itop
        real(kind=8), allocatable, target :: sten(:,:,:)
        real(kind=8) :: tot_vol
        integer :: i, j, k
        allocate(sten(3,3,nzmax))
        do k = 1, nzmax
          tot_vol = 0.0d0
          do i = 1, 3
            do j = 1, 3
              sten(i,j,k) = kappa_pd(ivent-2+i, jvent-2+j, k)
              tot_vol = tot_vol + kappa_pd(ivent-2+i, jvent-2+j, k)
            enddo
          enddo
          sten(:,:,k) = sten(:,:,k)/tot_vol
        enddo
        call B200_Check(a3g_set_umbrella(b200_ctx, int(ivent, c_int32_t), int(jvent, c_int32_t), &
                        int(ibase, c_int32_t), int(itop, c_int32_t), c_loc(sten)), "a3g_set_umbrella")
        deallocate(sten)
      end subroutine B200_SetUmbrella

      ! In place of the umbrella block of MesoInterpolater (src/MesoInterpolater.f90:
      ! 233-248): after B200_SetWinds / B200_InterpWinds, while TimeNow < e_EndTime(1),
      ! call umbrella_winds(first_time) on the host and pass its field (it is the
      ! same on every level ibase..itop).
      subroutine B200_AddUmbrellaWinds
        use mesh,            only : nxmax, nymax
        use Source_Umbrella, only : uvx_pd, uvy_pd, ibase
        real(kind=8), allocatable, target :: ux(:,:), uy(:,:)
        allocate(ux(nxmax,nymax), uy(nxmax,nymax))
        ux = uvx_pd(1:nxmax,1:nymax,ibase)
        uy = uvy_pd(1:nxmax,1:nymax,ibase)
        call B200_Check(a3g_add_umbrella_winds(b200_ctx, 1_c_int32_t, int(nxmax, c_int32_t), 1_c_int32_t, &
                        int(nymax, c_int32_t), c_loc(ux), c_loc(uy)), "a3g_add_umbrella_winds")
        deallocate(ux, uy)
      end subroutine B200_AddUmbrellaWinds

      ! In place of the smoothing and 3x3 insertion of src/Ash3d.F90:446-458, after
      ! TephraSourceNodes and TephraSourceNodes_Umbrella.
      subroutine B200_AddSourceUmbrella
        use Source_Umbrella, only : SourceNodeFlux_Umbrella
        use time_data,       only : dt
        call B200_Check(a3g_add_source_umbrella(b200_ctx, c_loc(SourceNodeFlux_Umbrella), real(dt, c_double)), &
                        "a3g_add_source_umbrella")
      end subroutine B200_AddSourceUmbrella

      ! In place of the conversions of src/write_NETCDF.f90:3296-3298 (ashcon) and
      ! 3320-3330 (depocon, scaled and thresholded), before their nf90_put_var:
      ! the writer's own real(kind=op) buffers, op = 4, are filled on the device.
      subroutine B200_OutputAshcon(ashcon, depocon)
        real(c_float), intent(out), target, contiguous :: ashcon(:,:,:,:), depocon(:,:,:)
        call B200_Check(a3g_output_ashcon(b200_ctx, c_loc(ashcon), c_loc(depocon)), "a3g_output_ashcon")
      end subroutine B200_OutputAshcon

      ! NC_RestartFile_LoadConcen (src/write_NETCDF.f90:3701-3709), after its
      ! nf90_get_var calls: concen_pd(ts1) = ashcon, concen(ts0) = concen(ts1),
      ! outflow_xy1_pd = DepositGranularity = depocon, on the device.
      subroutine B200_RestartLoad(ashcon, depocon)
        real(c_float), intent(in), target, contiguous :: ashcon(:,:,:,:), depocon(:,:,:)
        call B200_Check(a3g_restart_load(b200_ctx, c_loc(ashcon), c_loc(depocon)), "a3g_restart_load")
      end subroutine B200_RestartLoad

      end module B200_Transport

!##############################################################################
! Drop-in replacements with the reference's names and signatures
!##############################################################################

      module AdvectionHorz
      use iso_c_binding
      use B200_Transport
      implicit none
      private
      public AdvectHorz
      contains
      subroutine AdvectHorz(itoggle)
        use mesh, only : ivent, jvent, kvent
        integer, intent(in) :: itoggle
        call B200_Check(a3g_advect_horz(b200_ctx, int(itoggle, c_int32_t), int(ivent, c_int32_t), &
                        int(jvent, c_int32_t), int(kvent, c_int32_t)), "AdvectHorz")
      end subroutine AdvectHorz
      end module AdvectionHorz

      module AdvectionVert_DCU
      use iso_c_binding
      use B200_Transport
      implicit none
      private
      public AdvectVert
      contains
      subroutine AdvectVert
        call B200_Check(a3g_advect_vert(b200_ctx), "AdvectVert")
      end subroutine AdvectVert
      end module AdvectionVert_DCU

      module Diffusion
      use iso_c_binding
      use B200_Transport
      implicit none
      private
      public Allocate_Diff, Deallocate_Diff, DiffuseHorz, DiffuseVert
      real(kind=8), public :: diffusivity_horz, diffusivity_vert
      real(kind=8), public :: Imp_fac = 0.5d0
      real(kind=8), public :: Imp_DT_fac = 4.0d0
      real(kind=8), dimension(:,:,:), pointer, public :: kx => null(), ky => null(), kz => null()
      contains
      subroutine Allocate_Diff   ! src/Diffusion.F90:83-104
        use mesh, only : nxmax, nymax, nzmax
        if(.not.associated(kx))allocate(kx(0:nxmax+1,0:nymax+1,0:nzmax+1)); kx = diffusivity_horz
        if(.not.associated(ky))allocate(ky(0:nxmax+1,0:nymax+1,0:nzmax+1)); ky = diffusivity_horz
        if(.not.associated(kz))allocate(kz(0:nxmax+1,0:nymax+1,0:nzmax+1)); kz = diffusivity_vert
      end subroutine Allocate_Diff
      subroutine Deallocate_Diff
        if(associated(kx)) deallocate(kx)
        if(associated(ky)) deallocate(ky)
        if(associated(kz)) deallocate(kz)
      end subroutine Deallocate_Diff
      subroutine DiffuseHorz(i)
        integer :: i
        call B200_Check(a3g_diffuse_horz(b200_ctx, int(i, c_int32_t)), "DiffuseHorz")
      end subroutine DiffuseHorz
      subroutine DiffuseVert
        call B200_Check(a3g_diffuse_vert(b200_ctx), "DiffuseVert")
      end subroutine DiffuseVert
      end module Diffusion

      subroutine Set_BC(bc_code)
        use iso_c_binding
        use B200_Transport
        integer, intent(in) :: bc_code
        call B200_Check(a3g_set_bc(b200_ctx, int(bc_code, c_int32_t)), "Set_BC")
      end subroutine Set_BC

      subroutine Adjust_DT(mesostep)
        use iso_c_binding
        use B200_Transport
        use io_data,   only : NextWriteTime
        use time_data, only : time, dt, dt_ip, dt_meso_next, Simtime_in_hours
        logical, intent(in), optional :: mesostep
        real(c_double) :: dtn
        logical :: meso
        meso = .false.
        if (present(mesostep)) meso = mesostep
        if (meso) then
          ! FAST_DT (src/Adjust_dt.f90:96-135): the maxima of the FP32 next met
          ! step, uploaded by B200_SetMetSteps right after Read_NextMesoStep;
          ! MesoInterpolater keeps dt_meso_last and does the per-step
          ! interpolation (src/MesoInterpolater.f90:250-258) itself
          call B200_Check(a3g_adjust_dt_meso(b200_ctx, 1_c_int32_t, 0_c_int32_t, real(time, c_double), &
                          real(NextWriteTime, c_double), real(Simtime_in_hours, c_double), dtn), "Adjust_DT")
          dt = dtn
          dt_ip = dtn
          dt_meso_next = dt
        else
          call B200_Check(a3g_adjust_dt(b200_ctx, real(time, c_double), real(NextWriteTime, c_double), &
                          real(Simtime_in_hours, c_double), dtn), "Adjust_DT")
          dt = dtn
          dt_ip = dtn
        endif
      end subroutine Adjust_DT

      subroutine TimeStepTotals(itime)
        use iso_c_binding
        use B200_Transport
        use io_units
        use io_data,     only : OutputStep_Marker
        use solution,    only : aloft_vol, dep_vol, outflow_vol, tot_vol, mass_aloft, SourceCumulativeVol
        use time_data,   only : time, SimStartHour, Simtime_in_hours, BaseYear, useLeap
        use Output_Vars, only : CloudArea
        integer, intent(in) :: itime
        real(c_double), target :: out4(4)
        character(len=13) :: DateTime
        interface
          character (len=13) function HS_yyyymmddhhmm_since(HoursSince,byear,useLeaps)
            real(kind=8) :: HoursSince
            integer      :: byear
            logical      :: useLeaps
          end function HS_yyyymmddhhmm_since
        end interface
        call B200_Check(a3g_timestep_totals(b200_ctx, c_loc(out4), c_loc(mass_aloft)), "TimeStepTotals")
        aloft_vol = out4(1); dep_vol = out4(2); outflow_vol = out4(3); tot_vol = out4(4)
        ! the per-log-step line and progress.txt of src/TimeStepTotals.f90:69-82
        DateTime = HS_yyyymmddhhmm_since(time+SimStartHour, BaseYear, useLeap)
        do io=1,2;if(VB(io).le.verbosity_info)then
          write(outlog(io),'(6x,i6,a1,f11.3,3x,a,5f12.5,f13.1)') itime, OutputStep_Marker, time, DateTime, &
                SourceCumulativeVol, dep_vol, aloft_vol, outflow_vol, tot_vol, CloudArea
        endif;enddo
        open(unit=fid_progress, file='progress.txt', status='replace', action='write')
        write(fid_progress,*) real(time/Simtime_in_hours, kind=4)
        close(fid_progress)
        OutputStep_Marker = ' '
      end subroutine TimeStepTotals
