"""SFbox input files of the parity cases run through the reference's own
sources (oracle/_ref/sfref) and through this library's input reader.

One small system per lattice family of the hot path, with the boundary,
molecule and segment kinds each family takes.  Shared by the fixture
generator (make_reference_golden.py) and the parity tests.
"""

_SOLVENT_TAIL = """mol : water : composition : (W)1
mol : water : freedom : solvent
"""

INPUTS_COMB_BRANCHED_SIDE = """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 28
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -0.6
mon : A : chi - W : 0.9
mon : B : chi - W : 0.2
mol : comb : composition : @dend(2. (A)2, (B)3, (A)3[(B)1][(B)2](A)1, (A)2)
mol : comb : freedom : restricted
mol : comb : theta : 1.5
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
"""

INPUTS_CHARGED_1D = """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 30
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
lat : flat : bondlength : 3e-10
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : S : valence : -0.2
mon : S : epsilon : 5
mon : A : freedom : free
mon : A : valence : 0.5
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - W : 0.5
mon : A : chi - S : -1.0
mol : pol : composition : (A)20
mol : pol : freedom : free
mol : pol : phibulk : 0.001
mol : Na : composition : (Na)1
mol : Na : freedom : free
mol : Na : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
"""

INPUTS = {
    # Lat1DFlat1stO, the C1 system at reduced size: surface, frozen S
    "1d_flat_surface": """lat : flat : gradients : 1
lat : flat : n_layers : 30
lat : flat : geometry : flat
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.5
mon : A : chi - S : -1.0
mol : pol : composition : (A)21
mol : pol : freedom : free
mol : pol : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # the C1 system itself
    "1d_flat_c1": """lat : flat : gradients : 1
lat : flat : n_layers : 100
lat : flat : geometry : flat
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.5
mon : A : chi - S : -1.0
mol : pol : composition : (A)100
mol : pol : freedom : free
mol : pol : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # mirror2 above, lambda_chi != lambda, copolymer and restricted
    # homopolymer
    "1d_flat_mirror2": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 25
lat : flat : lambda : 0.25
lat : flat : lambda_chi : 0.2
lat : flat : lowerbound : mirror1
lat : flat : upperbound : mirror2
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 1.1
mon : B : chi - W : -0.2
mon : A : chi - B : 0.5
mol : ab : composition : (A)6(B)5(A)3
mol : ab : freedom : free
mol : ab : phibulk : 0.02
mol : h : composition : (B)9
mol : h : freedom : restricted
mol : h : theta : 2.5
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # a layer adjustment (SFbox allows it with mirror1 on both sides only)
    "1d_flat_layer_adjustment": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 19
lat : flat : lambda : 0.16666666666666667
lat : flat : layer_adjustment : 0.7
lat : flat : lowerbound : mirror1
lat : flat : upperbound : mirror1
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.9
mon : B : chi - W : 0.3
mol : ab : composition : (A)5(B)5
mol : ab : freedom : free
mol : ab : phibulk : 0.03
mol : h : composition : (A)8
mol : h : freedom : restricted
mol : h : theta : 1.5
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    "1d_flat_periodic": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 33
lat : flat : lambda : 0.25
lat : flat : lowerbound : periodic
lat : flat : upperbound : periodic
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - B : 0.5
mon : A : chi - W : 1.2
mon : B : chi - W : -0.2
mol : aba : composition : (A)4(B)9(A)4
mol : aba : freedom : restricted
mol : aba : theta : 6
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # Lat2DCyl1stO, the C2 system at reduced size
    "2d_cylinder": """lat : cyl : gradients : 2
lat : cyl : geometry : cylindrical
lat : cyl : n_layers_x : 20
lat : cyl : n_layers_y : 16
lat : cyl : lambda : 0.16666666666666667
lat : cyl : lowerbound_x : mirror1
lat : cyl : upperbound_x : mirror1
lat : cyl : lowerbound_y : mirror1
lat : cyl : upperbound_y : mirror1
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 1.6
mon : B : chi - W : 0.0
mol : AB : composition : (A)6(B)5
mol : AB : freedom : free
mol : AB : phibulk : 0.005
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # Lat2DCyl1stO with a core (offset), a surface and mirror2
    "2d_cylinder_core": """lat : cyl : gradients : 2
lat : cyl : geometry : cylindrical
lat : cyl : n_layers_x : 14
lat : cyl : n_layers_y : 11
lat : cyl : offset_first_layer_x : 2
lat : cyl : lambda : 0.2
lat : cyl : lowerbound_x : surface
lat : cyl : upperbound_x : mirror1
lat : cyl : lowerbound_y : mirror1
lat : cyl : upperbound_y : mirror2
mon : S : freedom : frozen
mon : S : frozen_range : 0,0;0,12
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.9
mon : A : chi - S : -0.8
mol : a : composition : (A)12
mol : a : freedom : free
mol : a : phibulk : 0.02
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # Lat2DFlat1stO with a surface, mirror2 and a restricted molecule
    "2d_flat_surface": """lat : sq : gradients : 2
lat : sq : geometry : flat
lat : sq : n_layers_x : 14
lat : sq : n_layers_y : 11
lat : sq : lambda : 0.16666666666666667
lat : sq : lowerbound_x : surface
lat : sq : upperbound_x : mirror1
lat : sq : lowerbound_y : mirror2
lat : sq : upperbound_y : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : 0,0;0,12
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -0.8
mon : A : chi - W : 0.9
mon : B : chi - W : 0.2
mol : AB : composition : (A)5(B)4(A)2
mol : AB : freedom : free
mol : AB : phibulk : 0.02
mol : h : composition : (B)7
mol : h : freedom : restricted
mol : h : theta : 3
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # Lat3D1stO periodic diblock melt, the C3 system at reduced size
    "3d_periodic_melt": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : n_layers_x : 9
lat : box : n_layers_y : 9
lat : box : n_layers_z : 9
mon : A : freedom : free
mon : B : freedom : free
mon : A : chi - B : 0.2
mol : AB : composition : (A)7(B)6
mol : AB : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # Lat3D1stO with mixed mirror1 / mirror2 / periodic bounds and a particle
    "3d_mirror_colloid": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : n_layers_x : 8
lat : box : n_layers_y : 7
lat : box : n_layers_z : 6
lat : box : lowerbound_x : mirror1
lat : box : upperbound_x : mirror2
lat : box : lowerbound_y : mirror2
lat : box : upperbound_y : mirror1
lat : box : lowerbound_z : periodic
lat : box : upperbound_z : periodic
mon : S : freedom : frozen
mon : S : frozen_range : 1,1,2;2,2,4
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.5
mon : A : chi - W : 0.7
mon : B : chi - W : 0.2
mol : AB : composition : (A)5(B)4
mol : AB : freedom : free
mol : AB : phibulk : 0.02
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # Lat3D2ndO grafted brush, the C5 system at reduced size
    "3d_2nd_brush": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : n_layers_x : 6
lat : box : n_layers_y : 6
lat : box : n_layers_z : 8
lat : box : lowerbound_x : mirror1
lat : box : upperbound_x : mirror1
lat : box : lowerbound_y : mirror1
lat : box : upperbound_y : mirror1
lat : box : lowerbound_z : mirror1
lat : box : upperbound_z : mirror1
sys : noname : matrix_approach : second_order
mon : X : freedom : pinned
mon : X : pinned_range : =(1,1,1)(3,4,1)(5,2,1)(6,6,1)
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.3
mon : X : chi - W : 0.3
mon : A : Pf - A : 0.5
mol : brush : composition : (X)1(A)14
mol : brush : freedom : restricted
mol : brush : theta : 60
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # 3D FCC and HEX lattices around a particle, periodic box
    "3d_fcc_colloid": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : latticetype : FCC
lat : box : n_layers_x : 8
lat : box : n_layers_y : 7
lat : box : n_layers_z : 6
mon : S : freedom : frozen
mon : S : frozen_range : 1,1,2;2,2,4
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.5
mon : A : chi - W : 0.7
mon : B : chi - W : 0.2
mol : AB : composition : (A)5(B)4
mol : AB : freedom : free
mol : AB : phibulk : 0.02
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # Lat1DCyl1stO and Lat1DSphere1stO
    "1d_cylinder": """lat : l : gradients : 1
lat : l : geometry : cylindrical
lat : l : n_layers : 22
lat : l : lambda : 0.16666666666666667
lat : l : lambda_chi : 0.2
lat : l : lowerbound : mirror1
lat : l : upperbound : mirror1
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - B : 0.3
mon : A : chi - W : 1.4
mon : B : chi - W : -0.1
mol : AB : composition : (A)7(B)6
mol : AB : freedom : free
mol : AB : phibulk : 0.02
mol : h : composition : (A)9
mol : h : freedom : restricted
mol : h : theta : 5
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    "1d_sphere_colloid": """lat : l : gradients : 1
lat : l : geometry : spherical
lat : l : n_layers : 18
lat : l : offset_first_layer : 3
lat : l : lambda : 0.16666666666666667
lat : l : lowerbound : surface
lat : l : upperbound : mirror2
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.4
mon : A : chi - W : 0.6
mol : A : composition : (A)16
mol : A : freedom : free
mol : A : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # lumped second order, Lat1D2ndO
    "1d_2nd_lumped": """lat : l : gradients : 1
lat : l : geometry : flat
lat : l : n_layers : 24
lat : l : lambda : 0.16666666666666667
lat : l : lowerbound : surface
lat : l : upperbound : mirror2
sys : noname : matrix_approach : second_order
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.2
mon : A : chi - W : 0.6
mon : A : Pf - A : 0.5
mol : A : composition : (A)15
mol : A : freedom : free
mol : A : phibulk : 0.02
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # lumped second order, Lat2D2ndO: mirror2/mirror1 in x, surface/mirror2 in y
    "2d_2nd_lumped": """lat : sq : gradients : 2
lat : sq : geometry : flat
lat : sq : n_layers_x : 11
lat : sq : n_layers_y : 9
lat : sq : lambda : 0.16666666666666667
lat : sq : lowerbound_x : mirror2
lat : sq : upperbound_x : mirror1
lat : sq : lowerbound_y : surface
lat : sq : upperbound_y : mirror2
sys : noname : matrix_approach : second_order
mon : S : freedom : frozen
mon : S : frozen_range : 0,0;12,0
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -0.6
mon : A : chi - B : 0.4
mon : A : chi - W : 1.0
mon : B : chi - W : 0.1
mon : A : Pf - A : 0.45
mon : A : Pf - B : 0.3
mol : AB : composition : (A)6(B)5
mol : AB : freedom : free
mol : AB : phibulk : 0.05
mol : h : composition : (B)7
mol : h : freedom : restricted
mol : h : theta : 4
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # curved second order: Lat1DCyl2ndO, Lat1DSphere2ndO, Lat2DCyl2ndO
    "1d_cyl_2nd": """lat : l : gradients : 1
lat : l : geometry : cylindrical
lat : l : n_layers : 20
lat : l : lambda : 0.16666666666666667
lat : l : lowerbound : mirror1
lat : l : upperbound : mirror1
sys : noname : matrix_approach : second_order
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - B : 0.3
mon : A : chi - W : 1.3
mon : B : chi - W : -0.1
mon : A : Pf - A : 0.5
mon : A : Pf - B : 0.3
mol : AB : composition : (A)8(B)6
mol : AB : freedom : free
mol : AB : phibulk : 0.03
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    "1d_sphere_2nd": """lat : l : gradients : 1
lat : l : geometry : spherical
lat : l : n_layers : 16
lat : l : offset_first_layer : 4
lat : l : lambda : 0.16666666666666667
lat : l : lowerbound : surface
lat : l : upperbound : mirror2
sys : noname : matrix_approach : second_order
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.2
mon : A : chi - W : 0.5
mon : A : Pf - A : 0.45
mol : A : composition : (A)12
mol : A : freedom : free
mol : A : phibulk : 0.01
mol : r : composition : (A)7
mol : r : freedom : restricted
mol : r : theta : 20
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    "2d_cyl_2nd": """lat : cyl : gradients : 2
lat : cyl : geometry : cylindrical
lat : cyl : n_layers_x : 10
lat : cyl : n_layers_y : 8
lat : cyl : offset_first_layer_x : 2
lat : cyl : lambda : 0.16666666666666667
lat : cyl : lowerbound_x : surface
lat : cyl : upperbound_x : mirror1
lat : cyl : lowerbound_y : surface
lat : cyl : upperbound_y : mirror2
sys : noname : matrix_approach : second_order
mon : S : freedom : frozen
mon : S : frozen_range : 0,0;0,9
mon : T : freedom : frozen
mon : T : frozen_range : 1,0;11,0
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -0.7
mon : A : chi - B : 0.5
mon : A : chi - W : 1.1
mon : B : chi - W : 0.2
mon : A : Pf - A : 0.4
mol : AB : composition : (A)5(B)6
mol : AB : freedom : free
mol : AB : phibulk : 0.04
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # 3D HEX (periodic) and stencils lattices
    "3d_hex_colloid": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : latticetype : HEX
lat : box : n_layers_x : 8
lat : box : n_layers_y : 7
lat : box : n_layers_z : 6
mon : S : freedom : frozen
mon : S : frozen_range : 1,1,2;2,2,4
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.5
mon : A : chi - W : 0.7
mon : B : chi - W : 0.2
mol : AB : composition : (A)5(B)4
mol : AB : freedom : free
mol : AB : phibulk : 0.02
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    "3d_stencils_colloid": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : latticetype : stencils
lat : box : lambda0 : 0.1
lat : box : lambda1 : 0.08
lat : box : lambda2 : 0.02
lat : box : lambda3 : 0.0225
lat : box : n_layers_x : 8
lat : box : n_layers_y : 7
lat : box : n_layers_z : 6
lat : box : lowerbound_x : mirror1
lat : box : upperbound_x : mirror2
lat : box : lowerbound_y : mirror2
lat : box : upperbound_y : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : 1,1,2;2,2,4
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.5
mon : A : chi - W : 0.7
mon : B : chi - W : 0.2
mol : AB : composition : (A)5(B)4
mol : AB : freedom : free
mol : AB : phibulk : 0.02
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # overflow protection: the log-space Lat1DFlat1stOS and Lat2DCyl1stOS
    "1d_flat_overflow": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 30
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror2
sys : noname : overflow_protection : true
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.5
mon : A : chi - S : -1.0
mol : pol : composition : (A)21
mol : pol : freedom : free
mol : pol : phibulk : 0.01
mol : r : composition : (A)9
mol : r : freedom : restricted
mol : r : theta : 2
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    "2d_cyl_overflow": """lat : cyl : gradients : 2
lat : cyl : geometry : cylindrical
lat : cyl : n_layers_x : 12
lat : cyl : n_layers_y : 10
lat : cyl : lambda : 0.16666666666666667
lat : cyl : lowerbound_x : mirror1
lat : cyl : upperbound_x : mirror2
lat : cyl : lowerbound_y : mirror1
lat : cyl : upperbound_y : mirror2
sys : noname : overflow_protection : true
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 1.6
mon : B : chi - W : 0.0
mol : AB : composition : (A)6(B)5
mol : AB : freedom : free
mol : AB : phibulk : 0.005
mol : r : composition : (B)8
mol : r : freedom : restricted
mol : r : theta : 3
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # a symmetric dendrimer at a surface (SF_Dend1stO)
    "1d_dendrimer": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 24
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.0
mon : A : chi - W : 0.6
mon : B : chi - W : 0.2
mol : den : composition : @dend(2,(A)3,3,(B)2(A)1,2)
mol : den : freedom : restricted
mol : den : theta : 3
mol : lin : composition : (A)4(B)4
mol : lin : freedom : free
mol : lin : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # constant-force ensemble (mol : force) of a diblock at a surface
    "1d_force": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 26
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.2
mon : B : chi - W : 0.4
mol : AB : composition : (A)3(B)9
mol : AB : freedom : restricted
mol : AB : theta : 2
mol : AB : force : 0.3
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # second-order copolymer with a stiff range (SF_Copol2ndO_stiff_range)
    "3d_2nd_stiff_range": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : n_layers_x : 6
lat : box : n_layers_y : 5
lat : box : n_layers_z : 6
lat : box : lowerbound_x : mirror1
lat : box : upperbound_x : mirror1
lat : box : lowerbound_y : mirror1
lat : box : upperbound_y : mirror1
lat : box : lowerbound_z : mirror1
lat : box : upperbound_z : mirror1
lat : box : stiff_range : 1,1,1;3,5,6
sys : noname : matrix_approach : second_order
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.8
mon : B : chi - W : 0.1
mon : A : Pf - A : 0.6
mon : A : Pf - B : 0.4
mol : tri : composition : (A)4(B)5(A)3
mol : tri : freedom : restricted
mol : tri : theta : 20
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # a palindromic second-order copolymer (SF_Copol2ndO's symmetric route)
    "3d_2nd_palindrome": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : n_layers_x : 6
lat : box : n_layers_y : 5
lat : box : n_layers_z : 6
lat : box : lowerbound_x : mirror1
lat : box : upperbound_x : mirror2
lat : box : lowerbound_y : periodic
lat : box : upperbound_y : periodic
lat : box : lowerbound_z : mirror1
lat : box : upperbound_z : mirror1
sys : noname : matrix_approach : second_order
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.8
mon : B : chi - W : 0.1
mon : A : Pf - A : 0.6
mon : A : Pf - B : 0.4
mol : tri : composition : (A)4(B)5(A)4
mol : tri : freedom : restricted
mol : tri : theta : 20
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # branched copolymer (SF_Branched1stO) at an adsorbing surface: two
    # branch points, one with two side fragments ('][')
    "1d_branched": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 30
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.5
mon : B : chi - W : 1.2
mon : A : chi - S : -1.0
mol : pol : composition : (A)5[(B)3](A)4[(B)2][(A)3](B)6
mol : pol : freedom : free
mol : pol : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # a grafting-free restricted branched molecule next to a free linear one,
    # with a repeated branched group ((..[..]..)2)
    "1d_branched_restricted": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 24
lat : flat : lambda : 0.25
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror2
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.2
mon : A : chi - W : 0.4
mon : B : chi - W : 0.9
mol : br : composition : (A)3((A)2[(B)3](A)1)2(B)2
mol : br : freedom : restricted
mol : br : theta : 2.5
mol : lin : composition : (B)6
mol : lin : freedom : free
mol : lin : phibulk : 0.005
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # a branched diblock in a 2D cylinder
    "2d_branched": """lat : cyl : gradients : 2
lat : cyl : geometry : cylindrical
lat : cyl : n_layers_x : 14
lat : cyl : n_layers_y : 10
lat : cyl : lambda : 0.16666666666666667
lat : cyl : lowerbound_x : mirror1
lat : cyl : upperbound_x : mirror1
lat : cyl : lowerbound_y : mirror1
lat : cyl : upperbound_y : mirror1
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 1.4
mon : B : chi - W : 0.0
mol : AB : composition : (A)4[(A)3](B)5
mol : AB : freedom : free
mol : AB : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # a branched molecule around a 3D colloid
    "3d_branched": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : n_layers_x : 7
lat : box : n_layers_y : 6
lat : box : n_layers_z : 6
lat : box : lowerbound_x : mirror1
lat : box : upperbound_x : mirror1
lat : box : lowerbound_y : periodic
lat : box : upperbound_y : periodic
lat : box : lowerbound_z : mirror1
lat : box : upperbound_z : mirror2
mon : S : freedom : frozen
mon : S : frozen_range : 1,1,1;2,2,3
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1.0
mon : A : chi - W : 0.6
mon : B : chi - W : 0.3
mol : br : composition : (A)3[(B)2][(B)2](A)3
mol : br : freedom : free
mol : br : phibulk : 0.02
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # comb @dend(NA. main1, spacer, side, main2) (SF_Comb1stO)
    "1d_comb": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 30
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -0.8
mon : A : chi - W : 0.3
mon : B : chi - W : 0.8
mol : comb : composition : @dend(3. (A)4, (A)3, (B)4, (A)5)
mol : comb : freedom : free
mol : comb : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # homopolymer ring (mol : ring, SF_HomoRing1stO) at an adsorbing surface
    "1d_ring": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 30
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.5
mon : A : chi - S : -1.0
mol : pol : composition : (A)20
mol : pol : ring : true
mol : pol : freedom : free
mol : pol : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # asymmetric dendrimer @dend(G; S11, S12, ..., SG1, SG2) (SF_AsymDend1stO);
    # every generation's second fragment is (A)3 (see ASYM_MIXED below)
    "1d_asym_dendrimer": """lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 30
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.5
mon : B : chi - W : 1.2
mon : A : chi - S : -1.0
mol : den : composition : @dend(3; (A)2, (A)3, (A)1(B)2, (A)3, (A)2(B)1, (A)3)
mol : den : freedom : free
mol : den : phibulk : 0.01
""" + _SOLVENT_TAIL + """newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # charges (SF_Solve.cpp:164-177): a polyelectrolyte at a charged surface
    # with a 1:1 salt, the anion as neutralizer; Na and Cl share an iteration
    # variable class (equal chi) and differ by valence
    "1d_charged": INPUTS_CHARGED_1D,

    # charges with different dielectric constants of the liquid states
    # (E^2 terms), a restricted polyelectrolyte, mirror2 above, T = 310 K
    "1d_charged_eps": """sys : noname : temperature : 310
lat : flat : gradients : 1
lat : flat : geometry : flat
lat : flat : n_layers : 30
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror2
lat : flat : bondlength : 6e-10
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : S : valence : -0.4
mon : S : epsilon : 5
mon : A : freedom : free
mon : A : valence : 0.5
mon : A : epsilon : 20
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - W : 0.5
mon : A : chi - S : -1.0
mol : pol : composition : (A)20
mol : pol : freedom : restricted
mol : pol : theta : 1.5
mol : Na : composition : (Na)1
mol : Na : freedom : free
mol : Na : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # charges on the 1D cylinder around its axis (a charged diblock, salt,
    # the cation as neutralizer) and on a charged sphere with an offset
    # (liquid states of different epsilon)
    "1d_cyl_charged": """lat : l : gradients : 1
lat : l : geometry : cylindrical
lat : l : n_layers : 22
lat : l : lambda : 0.16666666666666667
lat : l : lowerbound : mirror1
lat : l : upperbound : mirror1
lat : l : bondlength : 4e-10
mon : A : freedom : free
mon : A : valence : -0.3
mon : B : freedom : free
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - B : 0.3
mon : A : chi - W : 1.4
mon : B : chi - W : -0.1
mol : AB : composition : (A)7(B)6
mol : AB : freedom : free
mol : AB : phibulk : 0.02
mol : Cl : composition : (Cl)1
mol : Cl : freedom : free
mol : Cl : phibulk : 0.01
mol : Na : composition : (Na)1
mol : Na : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    "1d_sphere_charged": """lat : l : gradients : 1
lat : l : geometry : spherical
lat : l : n_layers : 18
lat : l : offset_first_layer : 3
lat : l : lambda : 0.16666666666666667
lat : l : lowerbound : surface
lat : l : upperbound : mirror2
lat : l : bondlength : 5e-10
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : S : valence : 0.3
mon : A : freedom : free
mon : A : valence : -0.5
mon : A : epsilon : 40
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - S : -1.4
mon : A : chi - W : 0.6
mol : A : composition : (A)16
mol : A : freedom : free
mol : A : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : free
mol : Cl : phibulk : 0.02
mol : Na : composition : (Na)1
mol : Na : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # a comb whose side chains are branched (two fragments at one point)
    "1d_comb_branched_side": INPUTS_COMB_BRANCHED_SIDE,
    # charges on the 2D flat lattice (Lat2DFlat::ElectricPotential): a
    # charged surface row at lower x, mirrors elsewhere
    "2d_flat_charged": """lat : sq : gradients : 2
lat : sq : geometry : flat
lat : sq : n_layers_x : 14
lat : sq : n_layers_y : 11
lat : sq : lambda : 0.16666666666666667
lat : sq : lowerbound_x : surface
lat : sq : upperbound_x : mirror1
lat : sq : lowerbound_y : mirror2
lat : sq : upperbound_y : mirror1
lat : sq : bondlength : 3e-10
mon : S : freedom : frozen
mon : S : frozen_range : 0,1;0,11
mon : S : valence : -0.2
mon : S : epsilon : 5
mon : A : freedom : free
mon : A : valence : 0.5
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - W : 0.5
mon : A : chi - S : -1.0
mol : pol : composition : (A)12
mol : pol : freedom : free
mol : pol : phibulk : 0.002
mol : Na : composition : (Na)1
mol : Na : freedom : free
mol : Na : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # a charged corner: surfaces at lower x (row S) and lower y (column T),
    # the upper x row a surface too (U), different dielectric constants of
    # the liquid states; square, because SFbox checks the upper x surface
    # row at sites y + M - MX (Lat2DFlat.cpp:876-881)
    "2d_flat_charged_walls": """lat : sq : gradients : 2
lat : sq : geometry : flat
lat : sq : n_layers_x : 11
lat : sq : n_layers_y : 11
lat : sq : lambda : 0.16666666666666667
lat : sq : lowerbound_x : surface
lat : sq : upperbound_x : surface
lat : sq : lowerbound_y : surface
lat : sq : upperbound_y : mirror1
lat : sq : bondlength : 3e-10
mon : S : freedom : frozen
mon : S : frozen_range : 0,0;0,11
mon : S : valence : -0.1
mon : S : epsilon : 5
mon : T : freedom : frozen
mon : T : frozen_range : 1,0;11,0
mon : T : valence : 0.05
mon : T : epsilon : 10
mon : U : freedom : frozen
mon : U : frozen_range : 12,0;12,11
mon : A : freedom : free
mon : A : valence : -0.3
mon : A : epsilon : 60
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - W : 0.6
mon : A : chi - S : -0.5
mon : A : chi - T : -0.3
mol : pol : composition : (A)8
mol : pol : freedom : free
mol : pol : phibulk : 0.003
mol : Cl : composition : (Cl)1
mol : Cl : freedom : free
mol : Cl : phibulk : 0.01
mol : Na : composition : (Na)1
mol : Na : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # charges on the 2D cylinder with an offset (Lat2DCylinder::
    # ElectricPotential): a charged core surface at lower x
    "2d_cyl_charged": """lat : cyl : gradients : 2
lat : cyl : geometry : cylindrical
lat : cyl : n_layers_x : 14
lat : cyl : n_layers_y : 11
lat : cyl : offset_first_layer_x : 2
lat : cyl : lambda : 0.2
lat : cyl : lowerbound_x : surface
lat : cyl : upperbound_x : mirror1
lat : cyl : lowerbound_y : mirror1
lat : cyl : upperbound_y : mirror2
lat : cyl : bondlength : 3e-10
mon : S : freedom : frozen
mon : S : frozen_range : 0,1;0,11
mon : S : valence : -0.1
mon : A : freedom : free
mon : A : valence : 0.4
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - W : 0.6
mon : A : chi - S : -0.8
mol : a : composition : (A)10
mol : a : freedom : free
mol : a : phibulk : 0.002
mol : Na : composition : (Na)1
mol : Na : freedom : free
mol : Na : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # the 2D cylinder from its axis (no offset): the first interior row has
    # no inner neighbour; a charged diblock, salt, a surface at upper y
    "2d_cyl_charged_axis": """lat : cyl : gradients : 2
lat : cyl : geometry : cylindrical
lat : cyl : n_layers_x : 12
lat : cyl : n_layers_y : 10
lat : cyl : lambda : 0.16666666666666667
lat : cyl : lowerbound_x : mirror1
lat : cyl : upperbound_x : mirror1
lat : cyl : lowerbound_y : mirror1
lat : cyl : upperbound_y : surface
lat : cyl : bondlength : 4e-10
mon : S : freedom : frozen
mon : S : frozen_range : 1,11;12,11
mon : S : valence : 0.1
mon : S : epsilon : 8
mon : A : freedom : free
mon : A : valence : -0.3
mon : B : freedom : free
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - B : 0.3
mon : A : chi - W : 1.2
mon : B : chi - S : -0.6
mol : AB : composition : (A)6(B)5
mol : AB : freedom : free
mol : AB : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : free
mol : Cl : phibulk : 0.01
mol : Na : composition : (Na)1
mol : Na : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # charges with second-order propagators (Lat1D2ndO): a charged surface,
    # a semiflexible polyelectrolyte with salt and a neutralizer
    "1d_2nd_charged": """lat : l : gradients : 1
lat : l : geometry : flat
lat : l : n_layers : 24
lat : l : lambda : 0.16666666666666667
lat : l : lowerbound : surface
lat : l : upperbound : mirror2
lat : l : bondlength : 3e-10
sys : noname : matrix_approach : second_order
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : S : valence : -0.2
mon : A : freedom : free
mon : A : valence : 0.3
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - S : -1.2
mon : A : chi - W : 0.6
mon : A : Pf - A : 0.5
mol : A : composition : (A)15
mol : A : freedom : free
mol : A : phibulk : 0.002
mol : Na : composition : (Na)1
mol : Na : freedom : free
mol : Na : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # charges with the six-direction 3D second-order propagators (Lat3D2ndO)
    "3d_2nd_charged": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : n_layers_x : 6
lat : box : n_layers_y : 5
lat : box : n_layers_z : 6
lat : box : lowerbound_x : mirror1
lat : box : upperbound_x : mirror1
lat : box : lowerbound_y : periodic
lat : box : upperbound_y : periodic
lat : box : lowerbound_z : mirror2
lat : box : upperbound_z : mirror1
lat : box : bondlength : 3e-10
sys : noname : matrix_approach : second_order
mon : S : freedom : frozen
mon : S : frozen_range : 2,2,2;3,3,3
mon : S : valence : 0.3
mon : A : freedom : free
mon : A : valence : -0.2
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - S : -0.8
mon : A : chi - W : 0.5
mon : A : Pf - A : 0.4
mol : A : composition : (A)8
mol : A : freedom : free
mol : A : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : free
mol : Cl : phibulk : 0.01
mol : Na : composition : (Na)1
mol : Na : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
    # charges with overflow protection (the log-space Lat1DFlat1stOS)
    "1d_charged_overflow": INPUTS_CHARGED_1D.replace("lat : flat : bondlength : 3e-10\n",
                                                      "lat : flat : bondlength : 3e-10\nsys : noname : overflow_protection : true\n"),
    # charges on the 3D lattice (Lat3D::ElectricPotential): a charged
    # colloid inside a mirror / periodic box
    "3d_charged_colloid": """lat : box : gradients : 3
lat : box : geometry : flat
lat : box : n_layers_x : 8
lat : box : n_layers_y : 7
lat : box : n_layers_z : 6
lat : box : lowerbound_x : mirror1
lat : box : upperbound_x : mirror2
lat : box : lowerbound_y : mirror2
lat : box : upperbound_y : mirror1
lat : box : lowerbound_z : periodic
lat : box : upperbound_z : periodic
lat : box : bondlength : 3e-10
mon : S : freedom : frozen
mon : S : frozen_range : 1,1,2;2,2,4
mon : S : valence : -0.3
mon : S : epsilon : 5
mon : A : freedom : free
mon : A : valence : 0.2
mon : B : freedom : free
mon : W : freedom : free
mon : Na : freedom : free
mon : Na : valence : 1
mon : Cl : freedom : free
mon : Cl : valence : -1
mon : A : chi - S : -1.5
mon : A : chi - W : 0.7
mon : B : chi - W : 0.2
mol : AB : composition : (A)5(B)4
mol : AB : freedom : free
mol : AB : phibulk : 0.02
mol : Na : composition : (Na)1
mol : Na : freedom : free
mol : Na : phibulk : 0.01
mol : Cl : composition : (Cl)1
mol : Cl : freedom : neutralizer
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-12
start
""",
}

# An asymmetric dendrimer whose generations' second fragments differ: SFbox's
# SF_AsymDend1stO::ComputePhi walks the second arm of generation i < G after
# its recursive call for generation i + 1 has reassigned the member
# SegBlock1 (SF_AsymDend1stO.cpp:218-219, :270-272), so those arms take the
# segments of generation G's second fragment.  Its lnGN is the molecule's
# partition function and agrees; its profiles do not describe the molecule.
ASYM_MIXED = INPUTS["1d_asym_dendrimer"].replace(
    "@dend(3; (A)2, (A)3, (A)1(B)2, (A)3, (A)2(B)1, (A)3)", "@dend(2; (A)3, (A)2, (B)2, (B)3)")
